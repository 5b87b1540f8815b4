"""Charge conservation on the GPU (pic_charge_density, pic_gauss_residual,
pic_gauss_check) through the C ABI.

rho and G = div E - rho against the oracle's numpy restatement
(oracle.charge_density / oracle.gauss_residual, whose definition the CPU
tests pin on the reference's own outputs), and the conservation of G by the
GPU step itself: to FP64 rounding in the plain form, to FP32 level in the
mixed form (FP32 E and in-cell offsets, per-warp 2^-22 current quantum)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    return 0.0 if d == 0.0 else d / max(np.linalg.norm(b), 1e-300)


def golden_sim(pkg, precision):
    d = np.load(os.path.join(GOLDEN, "ref_small.npz"))
    cells = tuple(int(c) for c in d["cells"])
    h, tau = float(d["h"]), float(d["tau"])
    table = [(float(d[f"in_s{s}_q_m"]), float(d[f"in_s{s}_m"]), s) for s in range(3)]
    sim = pkg.PicSimulation(cells, tuple(c * h for c in cells), tau, table, precision=precision)
    for s in range(3):
        arrs = [d[f"in_s{s}_{k}"] for k in ("x", "y", "z", "px", "py", "pz")]
        assert sim.load_particles(s, *arrs) == arrs[0].size
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        sim.set_field(f, d[f"in_{f}"])
    return d, sim, cells, (h, h, h)


def oracle_rho(oracle_mod, sim, cells, h):
    xs, ys, zs, ms = [], [], [], []
    for s in range(sim.nspecies):
        p = sim.particles(s)
        xs.append(p["x"]); ys.append(p["y"]); zs.append(p["z"])
        ms.append(np.full(p["x"].size, sim.cfg.species[s].m))
    return oracle_mod.charge_density(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs),
                                     np.concatenate(ms), cells, h)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 1e-6)])
def test_charge_density_and_residual_match_oracle(pkg, oracle_mod, precision, tol):
    d, sim, cells, h = golden_sim(pkg, precision)
    with sim:
        for step in range(3):
            rho = sim.charge_density()
            ref = oracle_rho(oracle_mod, sim, cells, h)
            assert rel_l2(rho, ref) < tol, step
            G = sim.gauss_residual()
            Gref = oracle_mod.gauss_residual(sim.get_field("Ex"), sim.get_field("Ey"), sim.get_field("Ez"), rho,
                                             cells, h)
            assert rel_l2(G, Gref) < 1e-12, step
            sim.step(step + 1)


def test_plain_step_conserves_gauss_law_on_golden(pkg, oracle_mod):
    """The FP64 GPU step from the reference fixture's inputs keeps G to
    rounding, and G after step 4 matches G of the reference's own step 4."""
    d, sim, cells, h = golden_sim(pkg, "fp64")
    with sim:
        base = sim.gauss_check(set_baseline=True)
        assert base[0] == 0.0 and base[1] > 0
        for st in range(1, 5):
            sim.step(st)
            chk = sim.gauss_check()
            assert chk[0] < 1e-12 * base[3], (st, chk)
        P = d["step4_particles"]
        m = np.array([float(d[f"in_s{s}_m"]) for s in range(3)])[P[:, 1].astype(int)]
        rho4 = oracle_mod.charge_density(P[:, 2], P[:, 3], P[:, 4], m, cells, h)
        G4 = oracle_mod.gauss_residual(d["step4_Ex"], d["step4_Ey"], d["step4_Ez"], rho4, cells, h)
        assert rel_l2(sim.gauss_residual(), G4) < 1e-12


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_gauss_law_over_steps(pkg, precision, tol):
    """Config-0 species on 32x4x4 cells, fields from zero, 20 steps (drifting
    beam, thermal electrons): max |G - G0| relative to max |rho|."""
    cfg = pkg.configs.CONFIGS["c0"]
    cells, hh, tau, ppc = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"]
    lengths = tuple(c * hh for c in cells)
    with pkg.PicSimulation(cells, lengths, tau, pkg.configs.species_table(ppc), precision=precision) as sim:
        for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
            sim.init_species(i, ppc, s["drift"], s["vth"], seed=3 + i)
        base = sim.gauss_check(set_baseline=True)
        worst = 0.0
        for st in range(1, 21):
            sim.step(st)
            chk = sim.gauss_check()
            worst = max(worst, chk[0] / chk[1])
        assert worst < tol, worst
        assert base[3] > 0


def test_gauss_check_needs_baseline(pkg):
    with pkg.PicSimulation((4, 4, 4), (0.4, 0.4, 0.4), 0.02, [(-1.0, -0.1, 1)]) as sim:
        sim.init_species(0, 2, (0.0, 0.0, 0.0), 0.01, seed=1)
        with pytest.raises(pkg.PicError):
            sim.gauss_check()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_momentum_matches_particles(pkg, precision):
    d, sim, cells, h = golden_sim(pkg, precision)
    with sim:
        sim.step(1)
        P = sim.momentum()
        for s in range(3):
            p = sim.particles(s)
            M = sim.cfg.species[s].m / sim.cfg.species[s].q_m
            ref = M * np.array([p["px"].sum(), p["py"].sum(), p["pz"].sum()])
            np.testing.assert_allclose(P[s], ref, rtol=1e-12, atol=1e-15 * abs(M) * p["px"].size)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_long_run_conserves_particles_and_charge(pkg, precision, tol):
    """1000 steps of the c2 species on 128x32x32 cells (12.6M particles): the
    beam bunches, tiles overflow and the step rebins.  Regression: a rebin of
    one species could resize the outbox while later species' overflow
    leftovers were still in it, silently losing particles (found by the
    Gauss-law check).  Every species keeps its particles and G stays put."""
    cells, ppc = (128, 32, 32), 32
    cfg = dict(pkg.configs.CONFIGS["c2"], cells=cells, ppc=ppc)
    with pkg.PicSimulation(cells, tuple(c * cfg["h"] for c in cells), cfg["tau"], pkg.configs.species_table(ppc),
                           precision=precision) as sim:
        pkg.configs.init_config_species(sim, cfg, 0)
        n0 = [sim.num_particles(s) for s in range(3)]
        sim.gauss_check(set_baseline=True)
        sim.run(1000)
        assert [sim.num_particles(s) for s in range(3)] == n0
        g = sim.gauss_check()
        print(f"{precision}: 1000-step Gauss drift max|G - G0| / max|rho| = {g[0] / g[1]:.3e}")
        assert g[0] < tol * g[1], g
