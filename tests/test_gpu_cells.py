"""Per-cell particle views (pic_get_cell_particles, the counterpart of reading
a GPUCell back, gpucell.h:290-427) against the CPU oracle's per-cell lists,
through the C ABI, after a few steps of config 0 (plain FP64 form): every
interior cell of every species holds the oracle's particles (same set, within
1e-12), its slots lie in its tile's bin, and the per-cell counts add up."""
import numpy as np
import pytest

from test_gpu_parity import c0_pair

pytestmark = pytest.mark.gpu


def test_cell_views_match_oracle(pkg, oracle_mod):
    sim, orc = c0_pair(pkg, oracle_mod)
    for st in range(1, 6):
        sim.step(st)
        assert orc.step() == 0
    p = orc.particles()
    keys = ("x", "y", "z", "px", "py", "pz")
    NX, NY, NZ = sim.shape
    counts = np.zeros(NX * NY * NZ, np.int64)
    for s in range(sim.nspecies):
        sel = p["sort"] == s
        for i in range(NX - 2):
            for l in range(NY - 2):
                for k in range(NZ - 2):
                    cell = (i * NY + l) * NZ + k
                    v = sim.cell_particles(s, cell)
                    m = sel & (p["cell"] == cell)
                    got = np.stack([v[q] for q in keys], 1)
                    want = np.stack([p[q][m] for q in keys], 1)
                    assert got.shape == want.shape, (s, cell)
                    if got.shape[0]:
                        got = got[np.lexsort(got.T[::-1])]
                        want = want[np.lexsort(want.T[::-1])]
                        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
                        assert np.all(np.diff(v["slot"]) > 0) and v["slot"][0] >= v["bin_offset"]
                    counts[cell] += got.shape[0]
    assert np.array_equal(counts, sim.cell_counts())
    # a ghost cell is not a cell of the grid
    with pytest.raises(pkg.PicError):
        sim.cell_particles(0, (NX - 1) * NY * NZ)
    sim.close()
    orc.close()


def test_cell_view_fp32_form(pkg):
    """The FP32 form's view converts cell + offset to global positions and
    agrees with the species export."""
    cells, h, tau, ppc = (8, 4, 8), 0.1, 0.02, 6
    table = pkg.configs.species_table(ppc)
    with pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, table, precision="fp32") as sim:
        for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
            sim.init_species(i, ppc, s["drift"], max(s["vth"], 0.03), i + 1)
        sim.run(3)
        allp = sim.particles(1)
        NX, NY, NZ = sim.shape
        tot = 0
        for i in range(cells[0]):
            for l in range(cells[1]):
                for k in range(cells[2]):
                    cell = (i * NY + l) * NZ + k
                    v = sim.cell_particles(1, cell)
                    m = allp["cell"] == cell
                    assert v["x"].size == int(m.sum())
                    if v["x"].size:
                        a = np.sort(v["x"] + 10 * v["y"] + 100 * v["z"])
                        b = np.sort(allp["x"][m] + 10 * allp["y"][m] + 100 * allp["z"][m])
                        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
                    tot += v["x"].size
        assert tot == sim.num_particles(1)
