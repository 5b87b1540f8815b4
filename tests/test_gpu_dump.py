"""On-disk checkpoint / resume through the reference's dump format
(pic_dump_write / pic_dump_read): a run written after a few steps and read
into a fresh handle continues as the original does."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz")


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    return 0.0 if d == 0.0 else d / max(np.linalg.norm(b), 1e-300)


def make(pkg, precision):
    cfg = pkg.configs.CONFIGS["c0"]
    cells, h, tau, ppc = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"]
    sim = pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, pkg.configs.species_table(ppc),
                            precision=precision)
    return sim, cfg


def table(sim):
    rows = []
    for s in range(sim.nspecies):
        p = sim.particles(s)
        rows.append(np.stack([p["cell"].astype(float), np.full(p["x"].size, float(s)), p["x"], p["y"], p["z"],
                              p["px"], p["py"], p["pz"]], 1))
    t = np.concatenate(rows)
    return t[np.lexsort((t[:, 4], t[:, 3], t[:, 2], t[:, 1], t[:, 0]))]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_dump_resume_continues_the_run(pkg, tmp_path, precision, tol):
    a, cfg = make(pkg, precision)
    b, _ = make(pkg, precision)
    with a, b:
        for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
            a.init_species(i, cfg["ppc"], s["drift"], s["vth"], seed=30 + i)
        a.run(3)
        path = str(tmp_path / pkg.mumu_name(0, 3))
        a.dump_write(path)
        b.dump_read(path)
        for f in FIELDS:
            assert np.array_equal(b.get_field(f), a.get_field(f)), f
        ta, tb = table(a), table(b)
        assert ta.shape == tb.shape and np.array_equal(ta[:, :2], tb[:, :2])
        np.testing.assert_allclose(tb[:, 2:], ta[:, 2:], rtol=0, atol=1e-15 if precision == "fp64" else 1e-7)
        a.run(3)
        b.run(3)
        for f in FIELDS:
            assert rel_l2(b.get_field(f), a.get_field(f)) < tol, f
        assert np.array_equal(a.cell_counts(), b.cell_counts())


def test_dump_read_rejects_another_configuration(pkg, tmp_path):
    a, cfg = make(pkg, "fp64")
    with a:
        for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
            a.init_species(i, cfg["ppc"], s["drift"], s["vth"], seed=1 + i)
        path = str(tmp_path / "x.dat")
        a.dump_write(path)
    other = pkg.PicSimulation((8, 4, 4), (0.8, 0.4, 0.4), 0.02, pkg.configs.species_table(cfg["ppc"]))
    with other:
        with pytest.raises(pkg.PicError):
            other.dump_read(path)
