"""The stress configuration's pieces on the GPU (non-uniform density profile,
hot electrons, dt = 0.05): device counts equal the host profile counts, the
FP32 form tracks the FP64 form, charge stays conserved under heavy
migration, and the adjoint of the differentiable run still matches finite
differences on such data."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CELLS, H, TAU, PPC = (32, 16, 16), 0.1, 0.05, 12


def stress_cfg(pkg, ppc=PPC, cells=CELLS):
    return dict(pkg.configs.CONFIGS["c4"], cells=cells, ppc=ppc)


def make(pkg, precision, cfg=None, seed=20):
    cfg = cfg or stress_cfg(pkg)
    cells = cfg["cells"]
    sim = pkg.PicSimulation(cells, tuple(c * cfg["h"] for c in cells), cfg["tau"],
                            pkg.configs.species_table(cfg["ppc"]), precision=precision)
    pkg.configs.init_config_species(sim, cfg, seed)
    return sim


def test_profile_counts_on_device(pkg):
    cfg = stress_cfg(pkg)
    prof = dict(pkg.configs.C4_PROFILE, ppc_mean=PPC)
    expect = pkg.profile_counts(CELLS, prof)
    with make(pkg, "fp32", cfg) as sim:
        counts = sim.cell_counts().reshape(sim.shape)[:CELLS[0], :CELLS[1], :CELLS[2]]
        # ions and electrons follow the profile, the beam is uniform
        assert np.array_equal(counts, 2 * expect + PPC)
        assert sim.num_particles(0) == sim.num_particles(1) == int(expect.sum())


def test_stress_fp32_tracks_fp64_and_conserves_charge(pkg):
    sims = {p: make(pkg, p) for p in ("fp64", "fp32")}
    try:
        for s in sims.values():
            s.gauss_check(set_baseline=True)
        e = {p: s.run(40, energies=True) for p, s in sims.items()}
        tot64, tot32 = e["fp64"][:, 3], e["fp32"][:, 3]
        assert np.max(np.abs(tot32 - tot64) / np.abs(tot64)) < 1e-4
        c64, c32 = sims["fp64"].cell_counts(), sims["fp32"].cell_counts()
        assert c64.sum() == c32.sum()
        moved = sims["fp32"].counters()[0]
        assert moved > 0
        g64, g32 = sims["fp64"].gauss_check(), sims["fp32"].gauss_check()
        assert g64[0] < 1e-11 * g64[1], g64
        assert g32[0] < 1e-4 * g32[1], g32
    finally:
        for s in sims.values():
            s.close()


def test_stress_adjoint_matches_finite_differences(pkg):
    """The differentiable run on stress data (12 ppc mean on 32x16x16 cells,
    non-uniform ions/electrons, hot electrons): gradient of the window loss
    w.r.t. the beam drift against FP64 central differences."""
    cfg = stress_cfg(pkg)
    steps, window, K = 30, 10, 7
    loss = dict(field="Ex", window=window, species=2, drift=(0.2, 0.0, 0.0), vth=0.002)
    with make(pkg, "fp64", cfg) as sim:
        base = sim.particles(2)
        sim.forward(steps, K)
        g = sim.backward(**loss)
    keys = ("x", "y", "z", "px", "py", "pz")

    def L(eps):
        with make(pkg, "fp64", cfg) as s:
            b = {k: base[k].copy() for k in keys}
            b["px"] = b["px"] + eps
            s.load_particles(2, *[b[k] for k in keys])
            s.forward(steps, steps)
            return s.loss_value(field="Ex", window=window)

    eps = 1e-8
    fd = (L(eps) - L(-eps)) / (2 * eps)
    assert abs(g["d_drift"][0] - fd) / abs(fd) < 1e-3, (g["d_drift"][0], fd)
    with make(pkg, "fp32", cfg) as sim:
        sim.forward(steps, K)
        g32 = sim.backward(**loss)
    assert abs(g32["d_drift"][0] - fd) / abs(fd) < 1e-3, (g32["d_drift"][0], fd)


def test_stress_plain_matches_reference(pkg):
    """The FP64 plain form in the stress regime (c4's profile, hot electrons,
    dt 0.05) against the reference's own 10 steps (tests/golden/ref_stress.npz):
    identical per-cell counts every step, energies and final fields within
    1e-12."""
    import os
    from conftest import GOLDEN, stress_inputs
    d = np.load(os.path.join(GOLDEN, "ref_stress.npz"))
    cells, h, tau, ppc = tuple(int(c) for c in d["cells"]), float(d["h"]), float(d["tau"]), int(d["ppc"])
    lengths = tuple(c * h for c in cells)
    inputs = stress_inputs(pkg, cells, lengths, ppc, int(d["seed"]))
    table = [(q_m, m, sort) for sort, _, m, q_m in inputs]
    with pkg.PicSimulation(cells, lengths, tau, table, precision="fp64") as sim:
        for sort, arrs, _, _ in inputs:
            assert sim.load_particles(sort, *arrs) == arrs[0].size
        for st in range(1, int(d["steps"]) + 1):
            sim.step(st)
            assert np.array_equal(sim.cell_counts(), d[f"step{st}_counts"]), st
            assert sim.energy_reference() == pytest.approx(float(d[f"step{st}_energy"]), rel=1e-12), st
        for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"):
            ref = d[f"final_{f}"]
            err = np.linalg.norm(sim.get_field(f) - ref) / max(np.linalg.norm(ref), 1e-300)
            assert err <= 1e-12, (f, err)
