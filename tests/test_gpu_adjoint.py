"""Differentiable run (pic_forward / pic_backward) through the C ABI.

1. pic_forward is the same time step as pic_step: fields within 1e-12
   relative L2 and identical per-cell counts after the run (only the order of
   the FP64 current sums differs).
2. The adjoint gradient of L = sum over the last `window` steps of
   h^3 sum E_x^2 matches FP64 central finite differences along seeded random
   directions of the beam's initial momenta, and along the beam drift and
   thermal spread: relative error below 1e-3 (see the FD test for the choice
   of eps).
3. The gradient does not depend on the checkpoint interval (segments
   recomputed from different checkpoints give the same adjoint).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H, TAU = 0.1, 0.02
KEYS = ("x", "y", "z", "px", "py", "pz")


def make(pkg, cells=(16, 8, 8), ppc=4, precision="fp64", seed=11):
    sim = pkg.PicSimulation(cells, tuple(c * H for c in cells), TAU, pkg.configs.species_table(ppc),
                            precision=precision)
    for s, sp in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        sim.init_species(s, ppc, drift=sp["drift"], vth=sp["vth"], seed=seed + s)
    return sim


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    return 0.0 if d == 0.0 else d / max(np.linalg.norm(b), 1e-300)


BEAM = 2
STEPS, WINDOW = 30, 10
LOSS = dict(field="Ex", window=WINDOW, species=BEAM, drift=(0.2, 0.0, 0.0), vth=0.002)


def loss_with_beam(pkg, beam, precision="fp64"):
    with make(pkg, precision=precision) as sim:
        assert sim.load_particles(BEAM, *[beam[k] for k in KEYS]) == beam["x"].size
        sim.forward(STEPS, STEPS)
        return sim.loss_value(field="Ex", window=WINDOW)


def fd_along(pkg, base, dp, eps=1e-6, precision="fp64"):
    """central difference of L along the momentum perturbation dp (n, 3)"""
    vals = []
    for sgn in (1.0, -1.0):
        b = {k: base[k].copy() for k in KEYS}
        b["px"] = base["px"] + sgn * eps * dp[:, 0]
        b["py"] = base["py"] + sgn * eps * dp[:, 1]
        b["pz"] = base["pz"] + sgn * eps * dp[:, 2]
        vals.append(loss_with_beam(pkg, b, precision))
    return (vals[0] - vals[1]) / (2 * eps)


def test_forward_is_the_step(pkg):
    with make(pkg) as a, make(pkg) as b:
        a.forward(12, 5)
        b.run(12)
        for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz"):
            assert rel_l2(a.get_field(f), b.get_field(f)) < 1e-12, f
        assert np.array_equal(a.cell_counts(), b.cell_counts())
        hist = a.history()
        assert hist.shape == (12, 3) and np.all(hist[-1] > 0)
        ex = b.get_field("Ex").reshape(b.shape)[1:-1, 1:-1, 1:-1]
        np.testing.assert_allclose(hist[-1, 0], H ** 3 * np.sum(ex * ex), rtol=1e-12)
        # the state after pic_forward continues with pic_step
        a.run(3)
        b.run(3)
        assert rel_l2(a.get_field("Ex"), b.get_field("Ex")) < 1e-12


def test_gradient_matches_finite_differences(pkg):
    """The reference's zigzag relay point (CurrentToMesh, cell.h:1306-1422) jumps
    where a step switches between crossing one cell-centre plane (relay on the
    trajectory) and two (relay pinned to both planes), so L is piecewise
    smooth with small jumps.  A central difference whose +-eps interval holds
    a jump is off by jump / (2 eps), whatever eps; the chance of one grows
    with eps times the number of perturbed particles.  So: sparse random
    directions (64 beam particles each) at eps = 1e-6, and dense directions
    (every beam particle) at eps = 1e-8."""
    with make(pkg) as sim:
        base = sim.particles(BEAM)
        sim.forward(STEPS, 7)
        g = sim.backward(**LOSS)
        L0 = sim.loss_value(field="Ex", window=WINDOW)
    assert g["loss"] == L0
    n = base["x"].size
    assert g["d_p0"].shape == (n, 3)
    rng = np.random.default_rng(2024)
    errs = {}
    for q in range(4):
        v = np.zeros((n, 3))
        idx = rng.choice(n, 64, replace=False)
        v[idx] = rng.standard_normal((64, 3))
        ad = float(np.sum(g["d_p0"] * v))
        errs[f"sparse{q}"] = abs(fd_along(pkg, base, v, eps=1e-6) - ad) / abs(ad)
    for q in range(2):
        v = rng.standard_normal((n, 3))
        ad = float(np.sum(g["d_p0"] * v))
        errs[f"dense{q}"] = abs(fd_along(pkg, base, v, eps=1e-8) - ad) / abs(ad)
    # drift (x) and thermal spread: p0 = drift + vth xi
    e_x = np.zeros((n, 3))
    e_x[:, 0] = 1.0
    errs["drift"] = abs(fd_along(pkg, base, e_x, eps=1e-8) - g["d_drift"][0]) / abs(g["d_drift"][0])
    xi = np.stack([base["px"] - 0.2, base["py"], base["pz"]], axis=1) / 0.002
    errs["vth"] = abs(fd_along(pkg, base, xi, eps=1e-8) - g["d_vth"]) / abs(g["d_vth"])
    assert max(errs.values()) < 1e-3, errs


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gradient_independent_of_checkpoints(pkg, precision):
    """One level (K = 1, 7, 30) and two levels (pic_forward2: segments of 12
    or 30 steps with a sub-checkpoint every 4 or 7) give the same gradient."""
    grads = []
    for K, K2 in ((1, None), (7, None), (STEPS, None), (12, 4), (STEPS, 7)):
        with make(pkg, precision=precision) as sim:
            sim.forward(STEPS, K, K2)
            grads.append(sim.backward(**LOSS))
    # FP64 recomputes are reproducible to rounding; the FP32 form's recomputed
    # steps add the FP64 current in no fixed order, which can move an FP32 ulp
    tol = 1e-9 if precision == "fp64" else 1e-4
    for g in grads[1:]:
        assert rel_l2(g["d_p0"], grads[0]["d_p0"]) < tol
        np.testing.assert_allclose(g["d_drift"], grads[0]["d_drift"], rtol=tol)


def test_mixed_forward_is_the_step(pkg):
    """FP32 form: the fixed-order pass adds the current in FP64 without the
    product push's 2^-22 warp quantum, so fields agree to FP32 level."""
    with make(pkg, precision="fp32") as a, make(pkg, precision="fp32") as b:
        a.forward(12, 5)
        b.run(12)
        for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz"):
            assert rel_l2(a.get_field(f), b.get_field(f)) < 1e-4, f
        assert np.abs(a.cell_counts() - b.cell_counts()).sum() <= 4
        a.run(2)  # continues with the product step


def test_mixed_gradient_matches_fp64(pkg):
    """The FP32 adjoint (FP32 per particle, FP64 field adjoints) against the
    FP64 adjoint and FP64 central differences of the same loss."""
    grads, order = {}, {}
    for prec in ("fp64", "fp32"):
        with make(pkg, precision=prec) as sim:
            p = sim.particles(BEAM)
            if prec == "fp64":
                base = p
            # d_p0 rows follow the handle's bin order, which depends on its
            # tiling; the bins keep the generation order inside a cell, so a
            # stable sort by cell gives one order for both forms
            order[prec] = np.argsort(p["cell"], kind="stable")
            sim.forward(STEPS, 7)
            grads[prec] = sim.backward(**LOSS)
    g64, g32 = grads["fp64"], grads["fp32"]
    assert abs(g32["loss"] - g64["loss"]) / g64["loss"] < 1e-4
    assert abs(g32["d_drift"][0] - g64["d_drift"][0]) / abs(g64["d_drift"][0]) < 1e-3
    assert abs(g32["d_vth"] - g64["d_vth"]) / abs(g64["d_vth"]) < 1e-3
    assert rel_l2(g32["d_p0"][order["fp32"]], g64["d_p0"][order["fp64"]]) < 1e-2
    n = base["x"].size
    e_x = np.zeros((n, 3))
    e_x[:, 0] = 1.0
    fd = fd_along(pkg, base, e_x, eps=1e-8)
    assert abs(g32["d_drift"][0] - fd) / abs(fd) < 1e-3


def test_frozen_branch_differences_match_adjoint(pkg):
    """Exact check of the adjoint along dense directions.  A forward that
    replays the recorded run's discrete choices (pic_forward_replay) is a
    smooth function of the initial momenta and the very map pic_backward
    differentiates; its central differences at eps 1e-6 must match the
    adjoint to differencing accuracy along the thermal spread, the drift and
    16 seeded random directions over every beam particle.  At eps = 0 the
    replay reproduces the recorded loss."""
    with make(pkg) as base:
        p0 = base.particles(BEAM)
        base.branch_record(True)
        base.forward(STEPS, 7)
        g = base.backward(**LOSS)
        n = p0["x"].size

        def loss(dp, eps):
            with make(pkg) as s:
                if eps:
                    s.perturb_momenta(BEAM, dp, eps)
                s.forward_replay(STEPS, base)
                return s.loss_value(field="Ex", window=WINDOW)

        assert abs(loss(None, 0.0) - g["loss"]) <= 1e-12 * abs(g["loss"])
        xi = np.stack([p0["px"] - 0.2, p0["py"], p0["pz"]], axis=1) / 0.002
        e_x = np.zeros((n, 3))
        e_x[:, 0] = 1.0
        dirs = {"vth": xi, "drift": e_x}
        # the 16 seeded dense directions over every beam particle (seeds 1..16)
        dirs.update({f"dense{k}": np.random.default_rng(k).standard_normal((n, 3)) for k in range(1, 17)})
        errs = {}
        for name, dp in dirs.items():
            eps = 1e-6
            fd = (loss(dp, eps) - loss(dp, -eps)) / (2 * eps)
            ad = float(np.sum(g["d_p0"] * dp))
            errs[name] = abs(fd - ad) / abs(ad)
        # central differences at eps 1e-6 of an FP64 loss carry rounding noise of
        # about 1e-16 |L| / eps, relative to a directional derivative that is
        # smaller along random directions (measured: 2e-9 .. 3e-6 over these 18)
        assert max(errs.values()) < 1e-5, errs
