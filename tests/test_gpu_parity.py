"""GPU parity of the plain FP64 form against the reference (golden fixtures
made by the reference's own functions) and the CPU oracle, through the C ABI.

Bar (plain form): identical per-cell particle counts and cell indices, E, B
and J within 1e-12 relative L2 per step.  Fields that involve no current sum
(the B half step) are bit-identical: the kernels are compiled without FMA
contraction.  J differs from the oracle only by the order of its sums
(shared/global atomics), hence the tolerance."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"]
REL = 1e-12   # relative L2, fields (plain form)
ABS_X = 1e-12  # absolute, particle positions / momenta after a few steps


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return 0.0 if d == 0.0 else d / max(nb, 1e-300)


def canon(tab):
    """rows (cell, sort, x, y, z, px, py, pz) sorted per cell by sort then position"""
    order = np.lexsort((tab[:, 4], tab[:, 3], tab[:, 2], tab[:, 1], tab[:, 0]))
    return tab[order]


def gpu_table(sim):
    rows = []
    for s in range(sim.nspecies):
        p = sim.particles(s)
        rows.append(np.stack([p["cell"].astype(np.float64), np.full(p["x"].size, float(s)), p["x"], p["y"], p["z"],
                              p["px"], p["py"], p["pz"]], axis=1))
    return canon(np.concatenate(rows))


def assert_particles_close(gt, rt, atol=ABS_X):
    assert gt.shape == rt.shape
    assert np.array_equal(gt[:, 0], rt[:, 0])  # cell of every particle
    assert np.array_equal(gt[:, 1], rt[:, 1])
    np.testing.assert_allclose(gt[:, 2:], rt[:, 2:], rtol=0, atol=atol)


def small_sim(pkg, precision="fp64", **kw):
    d = np.load(os.path.join(GOLDEN, "ref_small.npz"))
    cells = tuple(int(c) for c in d["cells"])
    h, tau = float(d["h"]), float(d["tau"])
    table = [(float(d[f"in_s{s}_q_m"]), float(d[f"in_s{s}_m"]), s) for s in range(3)]
    sim = pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, table, precision=precision, **kw)
    for s in range(3):
        arrs = [d[f"in_s{s}_{k}"] for k in ("x", "y", "z", "px", "py", "pz")]
        assert sim.load_particles(s, *arrs) == arrs[0].size
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        sim.set_field(f, d[f"in_{f}"])
    return d, sim


def test_small_substeps_vs_reference(pkg):
    d, sim = small_sim(pkg)
    sim.substep("b_half")
    for f in ("Hx", "Hy", "Hz", "Qx", "Qy", "Qz"):
        assert np.array_equal(sim.get_field(f), d[f"sub_b_half_{f}"]), f
    sim.substep("stage_fields")
    sim.substep("push_deposit")
    for f in ("Jx", "Jy", "Jz"):
        assert rel_l2(sim.get_field(f), d[f"sub_write_j_{f}"]) <= REL, f
    sim.substep("migrate")
    assert_particles_close(gpu_table(sim), canon(d["sub_migrate_particles"]))
    sim.substep("j_fold")
    for f in ("Jx", "Jy", "Jz"):
        assert rel_l2(sim.get_field(f), d[f"sub_j_fold_{f}"]) <= REL, f
    sim.substep("b_complete")
    for f in ("Hx", "Hy", "Hz"):
        assert np.array_equal(sim.get_field(f), d[f"sub_b_complete_{f}"]), f
    sim.substep("e_update")
    for f in ("Ex", "Ey", "Ez"):
        assert rel_l2(sim.get_field(f), d[f"sub_e_update_{f}"]) <= REL, f
    sim.substep("e_ghosts")
    for f in ("Ex", "Ey", "Ez"):
        assert rel_l2(sim.get_field(f), d[f"sub_e_ghosts_{f}"]) <= REL, f


def test_small_steps_vs_reference(pkg):
    d, sim = small_sim(pkg)
    for st in range(1, int(d["steps"]) + 1):
        sim.step(st)
        assert np.array_equal(sim.cell_counts(), d[f"step{st}_counts"]), st
        for f in FIELDS:
            assert rel_l2(sim.get_field(f), d[f"step{st}_{f}"]) <= REL, (st, f)
        assert sim.energy_reference() == pytest.approx(float(d[f"step{st}_energy"]), rel=REL)
        if f"step{st}_particles" in d.files:
            assert_particles_close(gpu_table(sim), canon(d[f"step{st}_particles"]))


def c0_pair(pkg, oracle_mod, precision="fp64", seed=0, steps_cfg="c0", **kw):
    cfg = pkg.configs.CONFIGS[steps_cfg]
    cells, h, tau, ppc = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"]
    lengths = tuple(c * h for c in cells)
    table = pkg.configs.species_table(ppc)
    sim = pkg.PicSimulation(cells, lengths, tau, table, precision=precision, **kw)
    orc = oracle_mod.OracleSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], seed)
        sim.load_particles(i, *arrs)
        orc.add_particles(s["sort"], *arrs, table[i][1], s["q_m"])
    return sim, orc


def oracle_table(orc):
    p = orc.particles()
    return canon(np.stack([p["cell"].astype(np.float64), p["sort"].astype(np.float64), p["x"], p["y"], p["z"],
                           p["px"], p["py"], p["pz"]], axis=1))


def test_c0_ten_steps_vs_oracle(pkg, oracle_mod):
    sim, orc = c0_pair(pkg, oracle_mod)
    d = np.load(os.path.join(GOLDEN, "ref_c0.npz"))
    for st in range(1, 11):
        sim.step(st)
        assert orc.step() == 0
        counts = sim.cell_counts()
        assert np.array_equal(counts, orc.cell_counts()), st
        assert np.array_equal(counts, d[f"step{st}_counts"]), st
        for f in FIELDS:
            assert rel_l2(sim.get_field(f), orc.get_field(f)) <= REL, (st, f)
        assert sim.energy_reference() == pytest.approx(orc.energy_reference(), rel=REL)
        assert sim.energy_reference() == pytest.approx(float(d[f"step{st}_energy"]), rel=REL)
    assert_particles_close(gpu_table(sim), oracle_table(orc))
    # FP64 energy diagnostics agree with the oracle's
    np.testing.assert_allclose(sim.energy(), orc.energies(), rtol=1e-10)
    for f in FIELDS:
        assert rel_l2(sim.get_field(f), d[f"final_{f}"]) <= REL, f


def test_tile_overflow_rebins(pkg, oracle_mod):
    """Tiles with no spare slot: every net arrival overflows a tile, the step
    rebins and the result still matches the oracle."""
    cells, h, tau, ppc = (12, 4, 8), 0.1, 0.02, 6
    lengths = tuple(c * h for c in cells)
    table = pkg.configs.species_table(ppc)
    sim = pkg.PicSimulation(cells, lengths, tau, table, capacity_slack=1e-9, capacity_pad=0, tile=(4, 4, 4))
    orc = oracle_mod.OracleSim(cells, lengths, tau)
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        drift = (0.45, 0.3, -0.2)  # every species drifts across tiles
        arrs = pkg.host_species(cells, lengths, i, ppc, drift, 0.05, 9)
        sim.load_particles(i, *arrs)
        orc.add_particles(s["sort"], *arrs, table[i][1], s["q_m"])
    moved = 0
    for st in range(8):
        sim.step(st)
        moved += int(sim.counters()[0])
        assert orc.step() == 0
        assert np.array_equal(sim.cell_counts(), orc.cell_counts()), st
        for f in ("Ex", "Ey", "Ez", "Jx", "Jy", "Jz"):
            assert rel_l2(sim.get_field(f), orc.get_field(f)) <= REL, (st, f)
    assert moved > 0
    assert_particles_close(gpu_table(sim), oracle_table(orc))


def test_stencil_violation_reported(pkg):
    """tau = 0.9 h lets a particle near c = 1 cross 0.9 of a cell in one step;
    the kernels check every stencil index and report PIC_ERR_STENCIL."""
    cells, h, tau = (4, 4, 4), 0.1, 0.09
    for precision in ("fp64", "fp32"):
        sim = pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, [(-1.0, -0.1, 1)], precision=precision)
        one = lambda v: np.array([v])  # noqa: E731
        sim.load_particles(0, one(0.19), one(0.15), one(0.15), one(40.0), one(0.0), one(0.0))
        with pytest.raises(pkg.PicError) as e:
            sim.step(1)
        assert e.value.status == -3


def test_device_generator_matches_host(pkg):
    cells, h, tau, ppc = (8, 4, 8), 0.1, 0.02, 5
    lengths = tuple(c * h for c in cells)
    sim = pkg.PicSimulation(cells, lengths, tau, pkg.configs.species_table(ppc))
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        sim.init_species(i, ppc, s["drift"], s["vth"], 4)
        host = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], 4)
        p = sim.particles(i)
        ht = canon(np.stack([np.zeros(host[0].size), np.zeros(host[0].size)] + host, axis=1))
        gt = canon(np.stack([np.zeros(p["x"].size), np.zeros(p["x"].size), p["x"], p["y"], p["z"], p["px"], p["py"],
                             p["pz"]], axis=1))
        assert np.array_equal(gt[:, 2:5], ht[:, 2:5])  # integer-derived uniforms: identical positions
        np.testing.assert_allclose(gt[:, 5:], ht[:, 5:], rtol=1e-12, atol=1e-15)
    counts = sim.cell_counts().reshape(10, 6, 10)
    assert np.all(counts[1:-1, 1:-1, 1:-1][:, :, :] >= 0)
    assert counts[:8, :4, :8].sum() == 3 * ppc * 8 * 4 * 8


def test_periodic_ghost_mode(pkg):
    """PIC_GHOSTS_PERIODIC adds the y passes the reference skips for Ex and Ez."""
    cells, h, tau = (5, 4, 6), 0.1, 0.02
    lengths = tuple(c * h for c in cells)
    sim = pkg.PicSimulation(cells, lengths, tau, [(-1.0, -0.1, 1)], ghosts="periodic")
    rng = np.random.default_rng(2)
    shape = tuple(c + 2 for c in cells)
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        sim.set_field(f, rng.normal(0, 1e-3, int(np.prod(shape))))
    sim.step(1)
    Nx, Ny, Nz = cells
    for f in ("Ex", "Ey", "Ez"):
        E = sim.get_field(f).reshape(shape)
        if f != "Ex":
            assert np.array_equal(E[0, 1:Ny, 1:Nz], E[Nx, 1:Ny, 1:Nz])
        if f != "Ez":
            assert np.array_equal(E[:Nx, :Ny, 0], E[:Nx, :Ny, Nz])
        if f != "Ey":
            assert np.array_equal(E[1:Nx, 0, 1:Nz], E[1:Nx, Ny, 1:Nz])


def test_mixed_form_tracks_plain(pkg, oracle_mod):
    """FP32 mixed form against the FP64 plain form from the same inputs:
    same physics, errors at FP32 level."""
    cfg = pkg.configs.CONFIGS["c0"]
    cells, h, tau, ppc = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"]
    lengths = tuple(c * h for c in cells)
    table = pkg.configs.species_table(ppc)
    sims = {p: pkg.PicSimulation(cells, lengths, tau, table, precision=p) for p in ("fp64", "fp32")}
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], 0)
        for sim in sims.values():
            sim.load_particles(i, *arrs)
    e = {p: sim.run(30, energies=True) for p, sim in sims.items()}
    tot64, tot32 = e["fp64"][:, 3], e["fp32"][:, 3]
    assert np.max(np.abs(tot32 - tot64)) / np.max(np.abs(tot64)) < 1e-4
    assert np.max(np.abs(e["fp32"][:, 0] - e["fp64"][:, 0])) / np.max(e["fp64"][:, 0]) < 1e-3
    c64, c32 = sims["fp64"].cell_counts(), sims["fp32"].cell_counts()
    assert c64.sum() == c32.sum()
    assert np.mean(c64 == c32) > 0.98
    for f in ("Ex", "Jx", "Hz"):
        a, b = sims["fp32"].get_field(f), sims["fp64"].get_field(f)
        assert rel_l2(a, b) < 1e-3, f


def test_mixed_centre_plane_ulp(pkg):
    """Offsets one float ulp below a cell-centre plane, moving by less than an
    ulp-scale step: the deposit must not see a centre crossing (regression:
    FP32 x + 2.5 rounds 0.49999997 up to the far side, and the split ratio
    divided by ~0)."""
    cells, h, tau = (4, 4, 4), 0.1, 0.02
    sim = pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, [(-1.0, -0.1, 1)], precision="fp32")
    below = np.nextafter(np.float32(0.5), np.float32(0.0))
    n = 6
    ref_cell = np.full(n, (1 * 6 + 1) * 6 + 1, np.int32)  # interior cell (1,1,1), reference numbering
    ox = np.full(n, below, np.float32)
    oy = np.array([below, 0.25, 0.75, below, 0.1, 0.9], np.float32)
    oz = np.full(n, np.float32(0.3))
    px = np.array([1e-9, 0.0, -1e-9, 1e-7, 0.01, -0.01], np.float32)
    py = np.array([0.0, 1e-9, 0.0, 1e-8, 0.0, 0.0], np.float32)
    pz = np.zeros(n, np.float32)
    assert sim.load_particles_cells(0, ref_cell, ox, oy, oz, px, py, pz) == n
    for st in range(3):
        sim.step(st)
    for f in ("Jx", "Jy", "Jz", "Ex", "Ey", "Ez"):
        assert np.isfinite(sim.get_field(f)).all(), f


def test_mixed_at_scale_stays_finite(pkg):
    """50M particles, 3 steps: fields and particles stay finite (the rare
    rounding paths only show up at this size)."""
    cells, ppc = (128, 64, 64), 32
    box = tuple(c * 0.1 for c in cells)
    sim = pkg.PicSimulation(cells, box, 0.02, pkg.configs.species_table(ppc), precision="fp32")
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        sim.init_species(i, ppc, s["drift"], s["vth"], i)
    n0 = sim.num_particles()
    sim.run(3)
    assert sim.num_particles() == n0
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz"):
        assert np.isfinite(sim.get_field(f)).all(), f
    e = sim.energy()
    assert np.isfinite(e).all() and e[2] > 0


def test_plasma_mirror_runs(pkg, oracle_mod):
    """The reference-shaped host surface (Plasma / Step / control points)."""
    P = pkg.Plasma(16, 4, 4, 1.6, 0.4, 0.4, 1.0, 8, 1.0 / 1836.0, 0.02)
    P.Initialize(host_generator=True)
    seen = []
    P.checker = lambda plasma, num, nt: seen.append((nt, num)) or (nt, num)
    P.Compute(3)
    assert [n for nt, n in seen if nt == 1] == [50, 270, 275, 400, 500, 550, 600]
    assert len(P.energy_history) == 3 and all(e >= 0 for _, e in P.energy_history)
