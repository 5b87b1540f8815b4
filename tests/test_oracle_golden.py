"""The CPU oracle (oracle/cpu_pic.c) against the golden fixtures produced by
the reference's own functions (tests/golden/make_golden.py).  Bit-exact:
the oracle restates the reference's arithmetic in the same order."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN

FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"]


def digest(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.float64:
        a = np.where(a == 0.0, 0.0, a)
    return hashlib.sha256(a.tobytes()).hexdigest()


def table(p):
    return np.stack([p["cell"].astype(np.float64), p["sort"].astype(np.float64), p["x"], p["y"], p["z"], p["px"],
                     p["py"], p["pz"]], axis=1)


def load_small(oracle_mod):
    d = np.load(os.path.join(GOLDEN, "ref_small.npz"))
    cells = tuple(int(c) for c in d["cells"])
    h, tau = float(d["h"]), float(d["tau"])
    sim = oracle_mod.OracleSim(cells, tuple(c * h for c in cells), tau)
    for sort in range(3):
        arrs = [d[f"in_s{sort}_{k}"] for k in ("x", "y", "z", "px", "py", "pz")]
        n = sim.add_particles(sort, *arrs, float(d[f"in_s{sort}_m"]), float(d[f"in_s{sort}_q_m"]))
        assert n == arrs[0].size
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        sim.set_field(f, d[f"in_{f}"])
    return d, sim


def test_small_substeps_bit_exact(oracle_mod):
    d, sim = load_small(oracle_mod)
    for sub in oracle_mod.SUBSTEPS:
        assert sim.substep(sub) == 0
        for f in FIELDS:
            key = f"sub_{sub}_{f}"
            if key in d.files:
                assert np.array_equal(sim.get_field(f), d[key]), key
        if sub == "migrate":
            assert np.array_equal(table(sim.particles()), d["sub_migrate_particles"])


def test_small_steps_bit_exact(oracle_mod):
    d, sim = load_small(oracle_mod)
    for st in range(1, int(d["steps"]) + 1):
        assert sim.step() == 0
        for f in FIELDS:
            assert np.array_equal(sim.get_field(f), d[f"step{st}_{f}"]), (st, f)
        assert np.array_equal(sim.cell_counts(), d[f"step{st}_counts"])
        assert sim.energy_reference() == float(d[f"step{st}_energy"])
        if f"step{st}_particles" in d.files:
            assert np.array_equal(table(sim.particles()), d[f"step{st}_particles"])


def test_c0_ten_steps_bit_exact(oracle_mod, pkg):
    d = np.load(os.path.join(GOLDEN, "ref_c0.npz"))
    cfg = pkg.configs.CONFIGS["c0"]
    cells, h, tau, ppc, seed = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"], int(d["seed"])
    lengths = tuple(c * h for c in cells)
    sim = oracle_mod.OracleSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    arrays = []
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], seed)
        arrays += arrs
        sim.add_particles(s["sort"], *arrs, pkg.configs.charge_weight(s["q_m"], s["density"], ppc), s["q_m"])
    # the generator is part of the fixture's definition
    assert digest(np.concatenate(arrays)) == str(d["inputs_digest"])
    for st in range(1, int(d["steps"]) + 1):
        assert sim.step() == 0
        assert np.array_equal(sim.cell_counts(), d[f"step{st}_counts"]), st
        assert sim.energy_reference() == float(d[f"step{st}_energy"]), st
        for f in FIELDS:
            assert digest(sim.get_field(f)) == str(d[f"step{st}_{f}_digest"]), (st, f)
        assert digest(table(sim.particles())) == str(d[f"step{st}_particles_digest"]), st
    for f in FIELDS:
        assert np.array_equal(sim.get_field(f), d[f"final_{f}"])


def test_golden_has_migration(oracle_mod):
    """The fixtures exercise cell-to-cell migration (counts change)."""
    d = np.load(os.path.join(GOLDEN, "ref_c0.npz"))
    c1, c10 = d["step1_counts"], d["step10_counts"]
    assert c1.sum() == c10.sum()
    assert not np.array_equal(c1, c10)


def test_oracle_matches_reference_live(oracle_mod, pkg):
    """Where the reference replay library exists (built from the reference
    sources), the oracle matches it bit for bit on fresh seeds and an odd grid."""
    if not oracle_mod.RefSim.available():
        pytest.skip("reference replay library not built here")
    cells, h, tau, ppc = (5, 3, 4), 0.1, 0.02, 5
    lengths = tuple(c * h for c in cells)
    sims = [oracle_mod.OracleSim(cells, lengths, tau), oracle_mod.RefSim(cells, lengths, tau)]
    rng = np.random.default_rng(11)
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        # faster beam so the zigzag branches with two segments occur often
        drift = (0.45, 0.2, -0.3) if s["name"] == "beam" else s["drift"]
        arrs = pkg.host_species(cells, lengths, i, ppc, drift, max(s["vth"], 0.05), 3)
        for sim in sims:
            sim.add_particles(s["sort"], *arrs, pkg.configs.charge_weight(s["q_m"], s["density"], ppc), s["q_m"])
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        a = rng.normal(0.0, 2e-2, sims[0].nodes)
        for sim in sims:
            sim.set_field(f, a)
    for st in range(6):
        for sim in sims:
            assert sim.step() == 0
        a, b = sims[0], sims[1]
        for f in FIELDS:
            assert np.array_equal(a.get_field(f), b.get_field(f)), (st, f)
        assert np.array_equal(table(a.particles()), table(b.particles())), st


def test_oracle_reports_cfl_violation(oracle_mod):
    """A particle moving more than half a cell in one step leaves the 5x5x5 tile
    range the reference can index; the oracle flags it instead of reading
    outside the tile."""
    # tau = 0.9 h: a particle near c = 1 crosses 0.9 of a cell per step
    cells, h, tau = (4, 4, 4), 0.1, 0.09
    sim = oracle_mod.OracleSim(cells, tuple(c * h for c in cells), tau)
    one = lambda v: np.array([v])  # noqa: E731
    sim.add_particles(1, one(0.19), one(0.15), one(0.15), one(40.0), one(0.0), one(0.0), -0.1, -1.0)
    rcs = [sim.substep(s) for s in oracle_mod.SUBSTEPS[:5]]
    assert rcs[4] == -3


def test_gauss_law_conserved_by_reference_outputs(oracle_mod):
    """The charge assignment of oracle.charge_density (linear weights on the
    cell-centre nodes, folded like the current) makes G = div E - rho a
    constant of the reference's own step: G from the fixture's inputs equals G
    after steps 1 and 4 of the reference (random initial E, all species)."""
    d = np.load(os.path.join(GOLDEN, "ref_small.npz"))
    cells = tuple(int(c) for c in d["cells"])
    h = (float(d["h"]),) * 3
    m_of = np.array([float(d[f"in_s{s}_m"]) for s in range(3)])
    xs = [np.concatenate([d[f"in_s{s}_{k}"] for s in range(3)]) for k in ("x", "y", "z")]
    ms = np.concatenate([np.full(d["in_s0_x"].size, m_of[0]), np.full(d["in_s1_x"].size, m_of[1]),
                         np.full(d["in_s2_x"].size, m_of[2])])
    rho0 = oracle_mod.charge_density(*xs, ms, cells, h)
    G0 = oracle_mod.gauss_residual(d["in_Ex"], d["in_Ey"], d["in_Ez"], rho0, cells, h)
    scale = np.abs(rho0).max()
    assert scale > 0 and np.abs(G0).max() > 0.1 * scale
    for st in (1, 4):
        P = d[f"step{st}_particles"]
        m = m_of[P[:, 1].astype(int)]
        rho = oracle_mod.charge_density(P[:, 2], P[:, 3], P[:, 4], m, cells, h)
        G = oracle_mod.gauss_residual(d[f"step{st}_Ex"], d[f"step{st}_Ey"], d[f"step{st}_Ez"], rho, cells, h)
        assert np.abs(G - G0).max() < 1e-12 * np.abs(G0).max(), st
        assert np.abs(rho - rho0).max() > 1e-6 * scale  # the charge did move


def test_charge_density_totals(oracle_mod):
    """rho on the interior nodes sums to the total charge (the fold keeps it)."""
    rng = np.random.default_rng(5)
    cells, h = (6, 5, 4), (0.1, 0.2, 0.3)
    L = [c * hh for c, hh in zip(cells, h)]
    x, y, z = (rng.uniform(0, l, 500) for l in L)
    m = rng.normal(0, 1, 500)
    r = oracle_mod.charge_density(x, y, z, m, cells, h).reshape(tuple(c + 2 for c in cells))
    np.testing.assert_allclose(r[1:-1, 1:-1, 1:-1].sum(), m.sum(), rtol=1e-12, atol=1e-12)


def test_quiet_default_run_bit_exact(oracle_mod, pkg):
    """The reference's own default run (main.cu:14: 100x4x4 cells, box
    1.1424 x 0.05 x 0.05, tau 0.001) from its own initial state (the
    library's quiet start, bit-identical to getUniformMaxwellianParticles):
    the C restatement reproduces the reference's 10 steps bit for bit on
    non-cubic cells with about 4000 particles per cell."""
    d = np.load(os.path.join(GOLDEN, "ref_quiet.npz"))
    cells = tuple(int(c) for c in d["cells"])
    sim = oracle_mod.OracleSim(cells, tuple(float(v) for v in d["lengths"]), float(d["tau"]),
                               threads=os.cpu_count() or 1)
    st = pkg.quiet_start()
    for s, name in enumerate(pkg.plasma.QUIET_SORTS):
        p = st[name]
        assert sim.add_particles(s, *[p[k] for k in ("x", "y", "z", "px", "py", "pz")], p["m"], p["q_m"]) == p["x"].size
    for step in range(1, int(d["steps"]) + 1):
        assert sim.step() == 0
        assert np.array_equal(sim.cell_counts(), d[f"step{step}_counts"]), step
        assert sim.energy_reference() == float(d[f"step{step}_energy"]), step
        if f"step{step}_Ex" in d.files:
            for f in FIELDS:
                assert np.array_equal(sim.get_field(f), d[f"step{step}_{f}"]), (step, f)
    tab = table(sim.particles())
    tab = tab[np.lexsort((tab[:, 4], tab[:, 3], tab[:, 2], tab[:, 1], tab[:, 0]))]
    assert tab.shape[0] == int(d["final_rows"])
    assert np.array_equal(tab[::int(d["sample"])], d["final_particles_sample"])


def test_stress_ten_steps_bit_exact(oracle_mod, pkg):
    """The stress regime (c4's density profile, cold ions, hot electrons of
    vth 0.1, dt 0.05; heavy migration) on 16x8x8 cells: the C restatement
    reproduces the reference's 10 steps bit for bit."""
    from conftest import stress_inputs
    d = np.load(os.path.join(GOLDEN, "ref_stress.npz"))
    cells, h, tau = tuple(int(c) for c in d["cells"]), float(d["h"]), float(d["tau"])
    lengths = tuple(c * h for c in cells)
    inputs = stress_inputs(pkg, cells, lengths, int(d["ppc"]), int(d["seed"]))
    assert digest(np.concatenate([a for _, arrs, _, _ in inputs for a in arrs])) == str(d["inputs_digest"])
    sim = oracle_mod.OracleSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    for sort, arrs, m, q_m in inputs:
        assert sim.add_particles(sort, *arrs, m, q_m) == arrs[0].size
    assert int(d["count_changes"]) > 1000  # the fixture migrates
    for st in range(1, int(d["steps"]) + 1):
        assert sim.step() == 0
        assert np.array_equal(sim.cell_counts(), d[f"step{st}_counts"]), st
        assert sim.energy_reference() == float(d[f"step{st}_energy"]), st
        for f in FIELDS:
            assert digest(sim.get_field(f)) == str(d[f"step{st}_{f}_digest"]), (st, f)
        assert digest(table(sim.particles())) == str(d[f"step{st}_particles_digest"]), st
