"""Benchmark of the B200 PIC time step: particle-steps/s.

Workload (default): 512x128x128 cells, 32 particles per cell per species,
3 species (805,306,368 particles), FP32 mixed form; synthetic seeded
uniform/Maxwellian inputs.  One "step" is one full PIC step (B half step,
push + deposit, migration, J fold, B completion, E update, E ghosts) over all
particles.  Inputs are larger than L2 (22.5 GB of particles), so no L2 flush
is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); the path has no exchange step on
one GPU's domain, so the ranks run independent replicas (different seeds),
"scaling": "weak"; value = all ranks' particle-steps / max-over-ranks time.

--impl reference times the reference's own CPU implementation (the reference's
functions compiled for the host, oracle/_ref) on the host cores at its own
CPU-runnable case (32x4x4 cells), rank 0 only.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s, FP32-mixed vs FP64 on B200 at stated error; adjoint/fwd time"
UNIT = "particle-steps/s"
# algorithmic bytes per particle-step of the push/deposit kernel: read + write
# of one particle (mixed: int32 cell + 3 FP32 offsets + 3 FP32 momenta = 28 B;
# plain: int32 cell + 3 FP64 positions + 3 FP64 momenta = 52 B)
BYTES_PER_PARTICLE_STEP = {"fp32": 56, "fp64": 104}
# algorithmic bytes per Yee cell-update: read E, B, J and write E, B
BYTES_PER_CELL_UPDATE = {"fp32": 72, "fp64": 120}
# DRAM bytes per particle of the push kernel (dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture of 50,331,648 particles, scaled to
# a launch by particle count since the kernel's traffic is proportional to it):
# profiles/push_mixed_128x64x64_ncu.md (2.830 GB) and
# profiles/push_plain_128x64x64_ncu.md (5.267 GB)
NCU_TRAFFIC_PER_PARTICLE = {"fp32": 2.830e9 / 50331648, "fp64": 5.267e9 / 50331648}
KERNELS_PER_STEP_NOTE = {
    "fp32": "push (forms the B half step of its staged tile), insert, clamp, j_fold x3, b_half twice in one pass, "
            "e_update, e_ghosts (both rounds in one launch); plus k_contribution_bound once per species after a load",
    "fp64": "b_half, push, insert, clamp, j_fold x3, b_complete, e_update, e_ghosts"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------- dist
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend: str | None = None):
        if self.world <= 1:
            return
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            torch.cuda.set_device(self.local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
        self.backend = backend
        self.pg = True

    def _t(self, x):
        import torch
        dev = "cuda" if getattr(self, "backend", "") == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def max(self, x: float) -> float:
        if not self.pg:
            return float(x)
        import torch.distributed as dist
        t = self._t(x)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return float(x)
        import torch.distributed as dist
        t = self._t(x)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            if getattr(self, "backend", "") == "nccl":
                dist.barrier(device_ids=[self.local])
            else:
                dist.barrier()

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()
            self.pg = False


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int | None = None):
        self.lines = []
        self.proc = None
        self.gpu_index = gpu_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(idx=int(f[0]), sm=float(f[1]), smax=float(f[2]), reasons=f[5:9]))
            except ValueError:
                continue
        if self.gpu_index is not None and any(r["idx"] == self.gpu_index for r in rows):
            rows = [r for r in rows if r["idx"] == self.gpu_index]
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r["reasons"]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------- our arm
def make_sim(pkg, cfg, form, device, seed_base):
    cells, h, tau, ppc = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"]
    box = tuple(c * h for c in cells)
    sim = pkg.PicSimulation(cells, box, tau, pkg.configs.species_table(ppc), precision=form, device=device)
    pkg.configs.init_config_species(sim, cfg, seed_base)
    return sim


def timed_steps(sim, K, torch):
    """K steps between CUDA events recorded on the library's stream."""
    stream = torch.cuda.ExternalStream(sim.lib.pic_stream(sim.h))
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    push_ms, b_ms, mig_ms, f2_ms, launches = [], [], [], [], 0
    t0.record(stream)
    for k in range(K):
        sim.step(k + 1)
        t = sim.timings()
        b_ms.append(float(t[0]))
        push_ms.append(float(t[1]))
        mig_ms.append(float(t[2]))
        f2_ms.append(float(t[3]))
        launches += int(sim.counters()[3])
    t1.record(stream)
    t1.synchronize()
    return t0.elapsed_time(t1), dict(b_half=b_ms, push=push_ms, migrate=mig_ms, fields2=f2_ms), launches


def run_ours(args, dist):
    import numpy as np
    import torch

    pkg = importlib.import_module("0buf_b200")
    cfg = workload_cfg(args, pkg.configs)
    form = args.form or cfg["precision"]
    dev = dist.local
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup
    seed_base = 1000 * dist.rank
    cells = cfg["cells"]
    ncell = int(np.prod(cells))

    sim = make_sim(pkg, cfg, form, dev, seed_base)
    n_local = sim.num_particles()
    sim.gauss_check(set_baseline=True)
    for w in range(W):
        sim.step(w + 1)
    dist.barrier()
    sampler = ClockSampler(dev) if dist.rank == 0 else None
    if sampler:
        sampler.start()
    elapsed_ms, phases, launches = timed_steps(sim, K, torch)
    clocks = sampler.stop() if sampler else None
    dist.barrier()
    t_max = dist.max(elapsed_ms)
    n_total = dist.sum(n_local)
    value = n_total * K / (t_max / 1e3)
    push_avg_ms = statistics.mean(phases["push"])
    yee_ms = statistics.mean(phases["b_half"]) + statistics.mean(phases["fields2"])
    layout = sim.layout()
    energy_last = sim.energy().tolist()
    state_last = {"energy": sim.energy(), "momentum": sim.momentum(), "gauss": sim.gauss_check()}
    sim.close()
    del sim

    peak, peak_kind = peaks()
    bpp = BYTES_PER_PARTICLE_STEP[form]
    achieved = bpp * n_local / (push_avg_ms / 1e3) / 1e9
    traffic = NCU_TRAFFIC_PER_PARTICLE[form]
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                "traffic": (round(traffic * n_local) if traffic else None),
                "kernel": f"k_push_{'mixed' if form == 'fp32' else 'plain'}",
                "algorithmic_bytes_per_launch": bpp * n_local, "avg_launch_ms": round(push_avg_ms, 4)}
    yee = {"cell_updates_per_s": round(ncell / (yee_ms / 1e3), 1), "ms_per_step": round(yee_ms, 4),
           "achieved_gbs": round(BYTES_PER_CELL_UPDATE[form] * ncell / (yee_ms / 1e3) / 1e9, 1)}
    yee["frac"] = round(yee["achieved_gbs"] / peak, 4)
    if form == "fp32":
        yee["note"] = ("J fold + both B half steps in one pass + E update + E ghosts; the first B half step is also "
                       "formed inside the push's staged field tile (its cost is in the push time)")

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": dist.world, "steps": K, "warmup": W,
        "ms_per_step": round(t_max / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if form == "fp32" else "f64", "data": "synthetic",
        "form": "FP32 mixed form (FP64 global J)" if form == "fp32" else "FP64 plain form",
        "config": workload_config(args, cfg, int(n_total / dist.world), dist.world),
        "roofline": roofline,
        "yee": yee,
        "phases_ms": {k: round(statistics.mean(v), 4) for k, v in phases.items()},
        "gpu_launches": launches,
        "launches_note": KERNELS_PER_STEP_NOTE[form],
        "energy_after": energy_last,
    }
    if clocks:
        out["clocks"] = clocks

    # end to end right after the main measurement: the later sections allocate
    # and free some 200 GB, and the driver has served multi-GB allocations
    # with 0.5 s stalls after such churn
    if not args.no_e2e:
        out["e2e"] = run_e2e(args, dist, pkg, cfg, form, torch, n_local)

    # FP64 plain form at the same configuration (N=1 only): the >= 2x claim,
    # and the FP32 form's error against this FP64 run from the same seed after
    # the same W + K steps (untimed steps fill up to W + K)
    if dist.world == 1 and not args.no_plain and form == "fp32":
        simp = make_sim(pkg, cfg, "fp64", dev, seed_base)
        simp.gauss_check(set_baseline=True)
        for w in range(2):
            simp.step(w + 1)
        Kp = max(3, K // 2)
        ms_p, ph_p, _ = timed_steps(simp, Kp, torch)
        for k in range(2 + Kp, W + K):
            simp.step(k + 1)
        vp = n_local * Kp / (ms_p / 1e3)
        pp = statistics.mean(ph_p["push"])
        out["plain_fp64"] = {"value": round(vp, 1), "ms_per_step": round(ms_p / Kp, 4), "steps": Kp,
                             "push_ms": round(pp, 4),
                             "push_achieved_gbs": round(104 * n_local / (pp / 1e3) / 1e9, 1),
                             "mixed_over_plain": round(value / vp, 3)}
        ref = {"energy": simp.energy(), "momentum": simp.momentum(), "gauss": simp.gauss_check()}
        out["accuracy"] = accuracy_vs_fp64(state_last, ref, W + K)
        simp.close()
        del simp
        if args.accuracy_steps > 0:
            out["accuracy_long"] = accuracy_history(pkg, cfg, dev, seed_base, args.accuracy_steps)

    if dist.world == 1 and not args.no_adjoint:
        out["adjoint"] = run_adjoint(args, pkg, dev)
    if dist.world == 1 and args.stress_adjoint:
        out["adjoint_stress"] = run_adjoint_stress(args, pkg, dev)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(args, cfg)
    return out


def accuracy_vs_fp64(s32, s64, steps):
    """FP32-form errors against the FP64 form after the same steps from the same
    seed: energies [E field, B field, kinetic, total] relative to the FP64
    total; total momentum per species relative to the largest per-species
    FP64 momentum |(m/q_m) sum p|; Gauss residual drift max |G - G0| over max |rho|."""
    import numpy as np
    e32, e64 = np.asarray(s32["energy"]), np.asarray(s64["energy"])
    p32, p64 = np.asarray(s32["momentum"]), np.asarray(s64["momentum"])
    tot = abs(e64[3])
    pscale = max(float(np.linalg.norm(p64, axis=1).max()), 1e-300)
    return {"steps": steps,
            "total_energy_rel_err": float(f"{abs(e32[3] - e64[3]) / tot:.3e}"),
            "field_E_energy_rel_err": float(f"{abs(e32[0] - e64[0]) / abs(e64[0]):.3e}"),
            "field_B_energy_rel_err": float(f"{abs(e32[1] - e64[1]) / max(abs(e64[1]), 1e-300):.3e}"),
            "kinetic_energy_rel_err": float(f"{abs(e32[2] - e64[2]) / abs(e64[2]):.3e}"),
            "momentum_rel_err": float(f"{float(np.linalg.norm(p32 - p64, axis=1).max()) / pscale:.3e}"),
            "gauss_drift_fp32": float(f"{s32['gauss'][0] / s32['gauss'][1]:.3e}"),
            "gauss_drift_fp64": float(f"{s64['gauss'][0] / s64['gauss'][1]:.3e}"),
            "note": "energies relative to the FP64 value (total energy: of the FP64 total); gauss drift = "
                    "max |G - G0| / max |rho|, G = div E - rho in FP64 on the device"}


def accuracy_history(pkg, cfg, dev, seed_base, steps):
    """Both forms from the same seed for `steps` steps, energies every step:
    the largest relative total-energy and field-energy errors over the run,
    and the final momentum and Gauss-residual errors."""
    import numpy as np
    hist, final = {}, {}
    for form in ("fp32", "fp64"):
        sim = make_sim(pkg, cfg, form, dev, seed_base)
        sim.gauss_check(set_baseline=True)
        hist[form] = sim.run(steps, energies=True)
        final[form] = {"energy": sim.energy(), "momentum": sim.momentum(), "gauss": sim.gauss_check()}
        sim.close()
    h32, h64 = hist["fp32"], hist["fp64"]
    out = accuracy_vs_fp64(final["fp32"], final["fp64"], steps)
    out["max_over_steps_total_energy_rel_err"] = float(f"{np.max(np.abs(h32[:, 3] - h64[:, 3]) / np.abs(h64[:, 3])):.3e}")
    out["max_over_steps_field_E_energy_rel_err"] = float(
        f"{np.max(np.abs(h32[:, 0] - h64[:, 0]) / np.maximum(np.abs(h64[:, 0]), 1e-300)):.3e}")
    out["total_energy_fp64_first_last"] = [float(h64[0, 3]), float(h64[-1, 3])]
    return out


ADJ_LOSS = dict(field="Ex", window=50, species=2, drift=(0.2, 0.0, 0.0), vth=0.002)


def match_particles(a, b, tol=1e-6):
    """Pairs the particles of two handles that hold the same generated
    particles (one FP64, one with FP32-rounded positions): index arrays ia,
    ib with a[ia[j]] ~ b[ib[j]].  Sorting by (cell, x, y, z) pairs all but the
    particles of one cell whose x lie within the FP32 rounding of each other;
    those cells are re-paired by nearest position.  Returns ia, ib and the
    number of re-paired particles."""
    import numpy as np
    ia = np.lexsort((a["z"], a["y"], a["x"], a["cell"]))
    ib = np.lexsort((b["z"], b["y"], b["x"], b["cell"]))
    pa = np.stack([a[k][ia] for k in ("x", "y", "z")], 1)
    pb = np.stack([b[k][ib] for k in ("x", "y", "z")], 1)
    bad = np.nonzero(np.max(np.abs(pa - pb), axis=1) > tol)[0]
    cells = np.unique(a["cell"][ia][bad])
    repaired = 0
    for c in cells:
        rows = np.nonzero(a["cell"][ia] == c)[0]
        d = np.sum((pa[rows, None, :] - pb[None, rows, :]) ** 2, axis=2)
        take = list(rows[np.argmin(d, axis=1)])
        if len(set(take)) == len(rows):  # a one-to-one nearest pairing
            ib[rows] = ib[take]
            pb[rows] = pb[take]
            repaired += int(np.sum(np.array(take) != rows))
    return ia, ib, repaired


def run_adjoint(args, pkg, dev):
    """The differentiable run at the adjoint configuration (128x32x32 cells,
    32 particles/cell/species, 300 steps, checkpoints every 25): device time of
    pic_forward and pic_backward in both forms, and the gradient of
    L = sum over the last 50 steps of h^3 sum E_x^2 against FP64 central
    differences of the FP64 forward -- along the beam drift and thermal spread
    (every beam particle moves: small eps, see below) and along random single-particle
    momentum directions (eps 1e-6).  Directions that move many particles at
    eps 1e-6 are not used: the reference's zigzag relay point makes L jump
    where a step changes from one to two crossed cell-centre planes, and such a
    difference measures the jump, not the gradient; the thermal-spread direction
    uses the median of three small eps for the same reason."""
    import numpy as np
    cfg = dict(pkg.configs.CONFIGS["c3"])
    if args.adjoint_cells:
        cfg["cells"] = tuple(int(c) for c in args.adjoint_cells.split(","))
    if args.adjoint_ppc:
        cfg["ppc"] = args.adjoint_ppc
    steps, K = (args.adjoint_steps or cfg["steps"]), 25
    out = {"config": f"c3: {'x'.join(map(str, cfg['cells']))} cells, {cfg['ppc']} particles/cell/species x 3, "
                     f"{steps} steps, checkpoints every {K}, loss = sum over the last 50 steps of h^3 sum E_x^2, "
                     "gradient w.r.t. the beam's initial momenta, drift and thermal spread"}
    import torch
    grads = {}
    base = None
    starts = {}
    # pic_step at the same configuration, timed the same way (CUDA events on
    # the library's stream): the comparison for the forward's per-step time
    step_ms = {}
    for form in ("fp64", "fp32"):
        sim = make_sim(pkg, cfg, form, dev, 0)
        for k in range(3):
            sim.step(k + 1)
        ms, _, _ = timed_steps(sim, 20, torch)
        step_ms[form] = ms / 20
        sim.close()
    for form in ("fp64", "fp32"):
        sim = make_sim(pkg, cfg, form, dev, 0)
        starts[form] = sim.particles(ADJ_LOSS["species"])
        if form == "fp64":
            base = starts[form]
        sim.forward(steps, K)
        g = sim.backward(**ADJ_LOSS)
        t = sim.adjoint_timings()
        sim.close()
        grads[form] = g
        out[form] = {"forward_ms": round(float(t[0]), 2), "backward_ms": round(float(t[1]), 2),
                     "backward_over_forward": round(float(t[1] / t[0]), 3),
                     "particle_steps_per_s_forward": round(sim_particles(cfg) * steps / (float(t[0]) / 1e3), 1),
                     "step_ms": round(step_ms[form], 4),
                     "forward_step_over_pic_step": round(float(t[0]) / steps / step_ms[form], 3),
                     "loss": g["loss"], "d_drift_x": float(g["d_drift"][0]), "d_vth": float(g["d_vth"])}
    # the FP64 gradient's own sensitivity to FP32 rounding: the FP64 adjoint
    # from the same initial state with every in-cell offset and momentum
    # rounded to FP32 (what the FP32 form starts from)
    sim = make_sim(pkg, cfg, "fp64", dev, 0)
    h = cfg["h"]
    for s in range(3):
        p = sim.particles(s)
        pos = np.stack([p["x"], p["y"], p["z"]], 1) / h
        cell = np.floor(pos)
        pos = (cell + (pos - cell).astype(np.float32).astype(np.float64)) * h
        mom = [p[k].astype(np.float32).astype(np.float64) for k in ("px", "py", "pz")]
        sim.load_particles(s, pos[:, 0], pos[:, 1], pos[:, 2], *mom)
    starts["fp64_r32"] = sim.particles(ADJ_LOSS["species"])
    sim.forward(steps, K)
    grads["fp64_r32"] = sim.backward(**ADJ_LOSS)
    sim.close()
    o64, o_r, _ = match_particles(starts["fp64"], starts["fp64_r32"])
    aligned = np.empty_like(grads["fp64"]["d_p0"])
    aligned[o64] = grads["fp64_r32"]["d_p0"][o_r]
    grads["fp64_r32"]["d_p0"] = aligned
    # dL/dp0 comes in each handle's own bin order, and the two forms tile the
    # grid differently: put the FP32 gradient in the FP64 particle order,
    # matching the same generated particles by (cell, x, y, z)
    o64, o32, repaired = match_particles(starts["fp64"], starts["fp32"])
    aligned = np.empty_like(grads["fp32"]["d_p0"])
    aligned[o64] = grads["fp32"]["d_p0"][o32]
    grads["fp32"]["d_p0"] = aligned
    out["fp32"]["p0_match"] = {"repaired_pairs": repaired, "max_dx": float(f"{max(np.max(np.abs(starts['fp64'][k][o64] - starts['fp32'][k][o32])) for k in ('x', 'y', 'z')):.3e}")}
    keys = ("x", "y", "z", "px", "py", "pz")

    def loss_of(dp, eps):
        vals = []
        for sg in (1.0, -1.0):
            sim = make_sim(pkg, cfg, "fp64", dev, 0)
            b = {k: base[k] for k in keys}
            for a, k in enumerate(("px", "py", "pz")):
                b[k] = base[k] + sg * eps * dp[:, a]
            sim.load_particles(ADJ_LOSS["species"], *[b[k] for k in keys])
            sim.forward(steps, steps)
            vals.append(sim.loss_value(field="Ex", window=ADJ_LOSS["window"]))
            sim.close()
        return (vals[0] - vals[1]) / (2 * eps)

    if args.no_fd:
        return out
    n = base["x"].size
    # run-to-run spread of L (FP64 atomics add the current in no fixed order)
    sim = make_sim(pkg, cfg, "fp64", dev, 0)
    sim.forward(steps, steps)
    out["loss_rerun_rel_diff"] = float(f"{abs(sim.loss_value(field='Ex', window=50) - grads['fp64']['loss']) / grads['fp64']['loss']:.3e}")
    sim.close()
    fd = {}
    e_x = np.zeros((n, 3))
    e_x[:, 0] = 1.0
    xi = np.stack([base["px"] - 0.2, base["py"], base["pz"]], axis=1) / ADJ_LOSS["vth"]
    d_drift = loss_of(e_x, 1e-8)
    # the spread direction moves every beam particle with random signs: its
    # signal is ~1000x below the drift's while it meets as many jumps, so take
    # the median of three small eps (one jump spoils at most one of them)
    vth_eps = (1e-9, 1e-10, 1e-11)
    vth_fd = [loss_of(xi, e) for e in vth_eps]
    d_vth = float(np.median(vth_fd))
    out["fd_vth_by_eps"] = {f"{e:g}": v for e, v in zip(vth_eps, vth_fd)}
    for form in ("fp64", "fp32"):
        g = grads[form]
        fd[form] = {"drift_rel_err": abs(g["d_drift"][0] - d_drift) / abs(d_drift),
                    "vth_rel_err": abs(g["d_vth"] - d_vth) / abs(d_vth), "particle_dirs_rel_err": []}
    rng = np.random.default_rng(16)
    canon = np.argsort(base["cell"], kind="stable")  # a tiling-independent particle order
    for _ in range(args.adjoint_dirs):
        v = np.zeros((n, 3))
        v[canon[rng.integers(n)]] = rng.standard_normal(3)
        f = loss_of(v, 1e-6)
        for form in ("fp64", "fp32"):
            ad = float(np.sum(grads[form]["d_p0"] * v))
            fd[form]["particle_dirs_rel_err"].append(abs(ad - f) / abs(f))
    for form in fd:
        errs = [fd[form]["drift_rel_err"], fd[form]["vth_rel_err"]] + fd[form]["particle_dirs_rel_err"]
        fd[form]["max_rel_err"] = max(errs)
        for k in list(fd[form]):
            v = fd[form][k]
            fd[form][k] = [float(f"{x:.3e}") for x in v] if isinstance(v, list) else float(f"{v:.3e}")
    out["fd_check"] = {"reference": "FP64 central differences of the FP64 forward", "fd_drift": d_drift,
                       "fd_vth": d_vth, **fd}
    out["fd_frozen"] = frozen_branch_check(pkg, cfg, dev, steps, base, grads)
    return out


def frozen_branch_check(pkg, cfg, dev, steps, base, grads):
    """Exact check of the adjoints along dense directions: FP64 central
    differences (eps 1e-7) of a forward that replays the discrete choices of
    a recorded FP64 run (pic_branch_record / pic_forward_replay) -- smooth in
    the initial momenta and the map pic_backward differentiates -- along the
    thermal spread, the drift and 16 seeded random directions over every beam
    particle."""
    import numpy as np
    rec = make_sim(pkg, cfg, "fp64", dev, 0)
    rec.branch_record(True)
    rec.forward(steps, steps)
    l_rec = rec.loss_value(field="Ex", window=ADJ_LOSS["window"])
    sp = ADJ_LOSS["species"]

    def loss(dp, eps):
        s = make_sim(pkg, cfg, "fp64", dev, 0)
        if eps:
            s.perturb_momenta(sp, dp, eps)
        s.forward_replay(steps, rec)
        v = s.loss_value(field="Ex", window=ADJ_LOSS["window"])
        s.close()
        return v

    n = base["x"].size
    xi = np.stack([base["px"] - ADJ_LOSS["drift"][0], base["py"], base["pz"]], axis=1) / ADJ_LOSS["vth"]
    e_x = np.zeros((n, 3))
    e_x[:, 0] = 1.0
    dirs = {"vth": xi, "drift_x": e_x}
    # 16 seeded dense directions over every beam particle (seeds 1..16), drawn
    # in a canonical particle order (by cell, generation order inside a cell:
    # a stable sort of the bins) so that they do not depend on the tiling
    canon = np.argsort(base["cell"], kind="stable")

    def dense(k):
        v = np.empty((n, 3))
        v[canon] = np.random.default_rng(k).standard_normal((n, 3))
        return v

    dirs.update({f"dense_{k}": dense(k) for k in range(1, 17)})
    out = {"reference": "FP64 central differences, eps 1e-7, of the forward replaying a recorded FP64 run's "
                        "discrete choices (taps, zigzag split classes, wraps, cell moves)",
           "replay_at_eps0_rel_diff": float(f"{abs(loss(None, 0.0) - l_rec) / abs(l_rec):.3e}")}
    # eps 1e-7: along the dense directions the directional derivative is ~1e-3
    # of the drift's and the third-order term of the 300-step map dominates at
    # eps 1e-6 (measured on the worst three: 9e-4, 2e-4, 2e-4 at 1e-6; 3e-6,
    # 4e-6, 1e-5 at 1e-7); rounding noise at 1e-7 stays near 1e-7 relative
    eps = 1e-7
    for name, dp in dirs.items():
        fd = (loss(dp, eps) - loss(dp, -eps)) / (2 * eps)
        out[name] = {"fd": fd}
        for form in ("fp64", "fp32"):
            ad = float(np.sum(grads[form]["d_p0"] * dp))
            out[name][f"{form}_adjoint"] = ad
            out[name][f"{form}_rel_err"] = float(f"{abs(ad - fd) / abs(fd):.3e}")
        if "fp64_r32" in grads:
            a64 = out[name]["fp64_adjoint"]
            ar = float(np.sum(grads["fp64_r32"]["d_p0"] * dp))
            out[name]["fp64_from_fp32_rounded_start_rel"] = float(f"{abs(ar - a64) / abs(a64):.3e}")
    for form in ("fp64", "fp32"):
        out[f"max_rel_err_{form}"] = max(v[f"{form}_rel_err"] for v in out.values() if isinstance(v, dict))
    if "fp64_r32" in grads:
        out["max_fp64_from_fp32_rounded_start_rel"] = max(
            v["fp64_from_fp32_rounded_start_rel"] for v in out.values() if isinstance(v, dict))
        out["rounded_start_note"] = ("the FP64 adjoint started from the same state rounded to FP32 (the FP32 form's "
                                     "start) moves by this much along each direction: the gradient's own sensitivity, "
                                     "a floor for any FP32 trajectory")
    out["directions"] = len(dirs)
    rec.close()
    return out


def run_adjoint_stress(args, pkg, dev):
    """The stress configuration's differentiable run at full size: FP32
    forward of 500 steps with two checkpoint levels (segments of 63 steps,
    a sub-checkpoint every 8) and the backward of the adjoint configuration's
    loss, checked against FP64 differences along the beam drift.

    The reference differences need a very small eps.  The hot electrons
    cross cell-centre planes all the time, and the zigzag deposit is
    continuous but not differentiable where a step starts or stops crossing
    one (kinks); its relay point even jumps where a step switches between
    crossing one plane and two.  Over 500 steps the perturbation grows, and
    with eps >= 1e-12 the +-eps interval holds such events (measured:
    central differences of 0.97, 0.58 and 0.24 at eps 1e-10, 1e-11 and
    1e-12, against about 0.45).  eps = 1e-13 is used: the central difference
    and both one-sided differences are reported, with the noise floor from
    two identical FP64 runs (the FP64 current is added in no fixed order)."""
    import numpy as np
    cfg = dict(pkg.configs.CONFIGS["c4"])
    steps, K, K2 = cfg["steps"], 63, 8
    sim = make_sim(pkg, cfg, "fp32", dev, 0)
    n = sim.num_particles()
    sim.forward(steps, K, K2)
    g = sim.backward(want_p0=False, **ADJ_LOSS)
    t = sim.adjoint_timings()
    sim.close()
    out = {"config": f"c4: {'x'.join(map(str, cfg['cells']))} cells, {n:,} particles, {steps} steps, FP32, "
                     f"checkpoints every {K} steps with sub-checkpoints every {K2}, loss of the adjoint configuration",
           "forward_ms": round(float(t[0]), 1), "backward_ms": round(float(t[1]), 1),
           "backward_over_forward": round(float(t[1] / t[0]), 3),
           "loss": g["loss"], "d_drift_x": float(g["d_drift"][0]), "d_vth": float(g["d_vth"])}
    if not args.no_fd:
        keys = ("x", "y", "z", "px", "py", "pz")
        ref = make_sim(pkg, cfg, "fp64", dev, 0)
        base = ref.particles(ADJ_LOSS["species"])
        ref.close()

        def loss_at(d):
            s = make_sim(pkg, cfg, "fp64", dev, 0)
            b = {k: base[k] for k in keys}
            b["px"] = base["px"] + d
            s.load_particles(ADJ_LOSS["species"], *[b[k] for k in keys])
            s.forward(steps, steps)
            v = s.loss_value(field="Ex", window=ADJ_LOSS["window"])
            s.close()
            return v

        eps = 1e-13
        l0, l0b, lp, lm = loss_at(0.0), loss_at(0.0), loss_at(eps), loss_at(-eps)
        central = (lp - lm) / (2 * eps)
        ad = float(g["d_drift"][0])
        out["fd_check"] = {"reference": "FP64 differences of the FP64 forward along the beam drift, eps 1e-13",
                           "central": central, "forward": (lp - l0) / eps, "backward": (l0 - lm) / eps,
                           "noise_floor": abs(l0b - l0) / (2 * eps),
                           "central_rel_err": float(f"{abs(ad - central) / abs(central):.3e}")}
    return out


def sim_particles(cfg) -> int:
    c = cfg["cells"]
    return int(c[0] * c[1] * c[2] * cfg["ppc"] * 3)


def run_e2e(args, dist, pkg, cfg, form, torch, n_local):
    """Same metric through the C ABI from pinned HOST memory, wall-clock timed
    around the whole public-API sequence: pic_create, the load of every
    species from pinned host arrays (host->device, 28 B per particle: int32
    cell + FP32 offsets and momenta), K x (pic_step + pic_energy, whose 32-byte
    result is read back to the host every step), pic_destroy."""
    import psutil

    need = 28 * n_local
    if psutil.virtual_memory().available < 2.5 * need:
        return {"value": None, "unit": UNIT, "note": f"host RAM below 2.5x the {need / 1e9:.1f} GB of inputs"}
    K = args.steps
    dev = dist.local
    sim = make_sim(pkg, cfg, form, dev, 1000 * dist.rank)
    host = []
    for s in range(sim.nspecies):
        n = sim.num_particles(s)
        arrs = [torch.empty(n, dtype=torch.int32, pin_memory=True)] + \
               [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(6)]
        got = sim.get_particles_cells(s, arrs)
        assert got == n
        host.append(arrs)
    table = pkg.configs.species_table(cfg["ppc"])
    box = tuple(c * cfg["h"] for c in cfg["cells"])
    sim.close()
    del sim
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    sim = pkg.PicSimulation(cfg["cells"], box, cfg["tau"], table, precision=form, device=dev)
    t1 = time.perf_counter()
    h2d = 0
    for s, arrs in enumerate(host):
        sim.load_particles_cells(s, *arrs)  # returns after its last copy and scatter
        h2d += sum(a.numel() * a.element_size() for a in arrs)
    t2 = time.perf_counter()
    energies = []
    for k in range(K):
        sim.step(k + 1)
        energies.append(sim.energy())  # the step's result, read back to the host
    t3 = time.perf_counter()
    sim.close()
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    ms = (t4 - t0) * 1e3
    phases = {"create": (t1 - t0) * 1e3, "load": (t2 - t1) * 1e3, "steps": (t3 - t2) * 1e3, "destroy": (t4 - t3) * 1e3}
    dist.barrier()
    t_max = dist.max(ms)
    n_total = dist.sum(n_local)
    return {"value": round(n_total * K / (t_max / 1e3), 1), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / K), "d2h_bytes_per_step": 32, "steps": K,
            "ms_total": round(t_max, 2), "phases_ms": {k: round(v, 1) for k, v in phases.items()},
            "phases_note": "this rank's wall clock per phase; the first step also sizes the outbox, and destroy "
                           "frees the load staging; after much allocation churn on a box a multi-GB device "
                           "allocation or free has taken the driver 0.5-0.9 s (in whichever phase makes it)",
            "path": "wall clock around pic_create + pic_load_particles_cells of every species from pinned host "
                    "memory + K x (pic_step + pic_energy read back to the host) + pic_destroy",
            "h2d_note": "the particles are loaded once; h2d_bytes_per_step is that load (28 B per particle) divided "
                        "by the K steps, so this figure depends on K"}


# ------------------------------------------------------- CPU baselines
# The reference's CPU path at the workload's density, on a periodic sub-box of
# 64x32x32 cells (1/128 of the 512x128x128 workload: 6.3M particles, 0.65 GB of
# the reference's 104-byte particles, well above the host caches).  Its
# containers (one 5000-particle array per cell, cell.h:55, 254) cannot hold the
# full workload.  Per-particle work is that of the full box: same species,
# density, dt and h, periodic.
REF_SAMPLE_CELLS = (64, 32, 32)


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    return importlib.import_module("oracle")


def species_of(cfg):
    """Species table rows (q_m, m, sort) and generator arguments of a
    configuration (plain data only: no product library is loaded)."""
    configs = importlib.import_module("0buf_b200.configs")
    sp = cfg.get("species") or configs.SPECIES_BEAM_PLASMA
    return configs.species_table(cfg["ppc"], sp), sp


NONUNIFORM_NOTE = ("the CPU path's generator (the oracle's restatement of the seeded device generator) covers the "
                   "uniform configurations c0-c3; this configuration's density profile is generated on the device "
                   "only, so the CPU figures are the uniform configurations' (cpu_baseline.configs)")


def uniform(cfg) -> bool:
    return not any("profile" in s for s in species_of(cfg)[1])


def cpu_sim(cfg, cells, threads, kind):
    """A CPU simulation of `cells` at the configuration's density: the
    reference's own functions (kind "reference", oracle/_ref) or the C
    restatement (kind "port"), inputs from the oracle's restated generator."""
    oracle = _oracle()
    table, sp = species_of(cfg)
    if any("profile" in s for s in sp):
        raise ValueError("CPU baselines cover the uniform configurations")
    h, tau, ppc = cfg["h"], cfg["tau"], cfg["ppc"]
    box = tuple(c * h for c in cells)
    if kind == "reference":
        sim = oracle.RefSim(cells, box, tau, threads=threads)
        for i, s in enumerate(sp):
            arrs = oracle.gen_species(cells, box, i, ppc, s["drift"], s["vth"], i, threads=threads)
            sim.add_particles(s["sort"], *arrs, table[i][1], s["q_m"])
    else:
        sim = oracle.OracleSim(cells, box, tau, threads=threads)
        for i, s in enumerate(sp):
            sim.init_species(s["sort"], i, ppc, s["drift"], s["vth"], i, table[i][1], s["q_m"])
    return sim


def cpu_time(cfg, cells, threads, kind, seconds, min_steps=1, max_steps=100000, warm=True):
    """Full PIC steps of the CPU path on `cells` with `threads` threads until
    `seconds` have passed (at least min_steps), after one untimed step unless
    warm is False.  The inputs are built with all host threads."""
    sim = cpu_sim(cfg, cells, cpu_threads(), kind)
    sim.set_threads(threads)
    n = sim.num_particles()
    if warm:
        assert sim.step() == 0
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and (steps < min_steps or time.perf_counter() - t0 < seconds):
        assert sim.step() == 0
        steps += 1
    dt = time.perf_counter() - t0
    sim.close()
    return {"value": round(n * steps / dt, 1), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{steps} steps of {cells[0]}x{cells[1]}x{cells[2]} cells ({n:,} particles), "
                      f"{threads} thread(s), {dt:.1f} s", "particles": n}


def ref_kind() -> str:
    return "reference" if _oracle().RefSim.available() else "port"


def cpu_baseline(args, cfg):
    """The reference CPU path on the box's host cores, rank 0 at N=1: the
    headline figure is the reference's own functions (oracle/_ref) on all
    cores on the workload's 64x32x32-cell sample; `configs` adds the C
    restatement (oracle/cpu_pic.c, bit-identical to the reference's
    functions) at the configurations c0, c3 (one thread and all cores) and
    c1 (all cores; one thread times one step when host RAM and time allow)."""
    import psutil
    configs = importlib.import_module("0buf_b200.configs")
    thr = cpu_threads()
    kind = ref_kind()
    if uniform(cfg):
        head = cpu_time(cfg, REF_SAMPLE_CELLS, thr, kind, args.cpu_seconds)
        head["sample"] += (f" -- a periodic sub-box of the {'x'.join(map(str, cfg['cells']))}-cell workload at its "
                           f"density; {'reference functions compiled for the host (oracle/_ref)' if kind == 'reference' else 'C restatement (oracle/cpu_pic.c)'}")
    else:
        head = {"value": None, "unit": UNIT, "note": NONUNIFORM_NOTE}
    out = dict(head)
    out["configs"] = {}
    runs = [("c0", "reference" if kind == "reference" else "port", thr, 4.0, True),
            ("c3", "port", 1, 0.0, False), ("c3", "port", thr, 2.0, True), ("c1", "port", thr, 0.0, True)]
    for name, k, t, secs, warm in runs:
        c = configs.CONFIGS[name]
        n = int(c["cells"][0] * c["cells"][1] * c["cells"][2]) * c["ppc"] * 3
        if psutil.virtual_memory().available < 200 * n:  # ~96 B per port particle plus tiles, with margin
            out["configs"][f"{name}_{t}t"] = {"value": None, "note": "host RAM"}
            continue
        r = cpu_time(c, c["cells"], t, k, secs, warm=warm)
        out["configs"][f"{name}_{t}t"] = r
    out["configs"]["c1_1t"] = {"value": None, "note": "not run by default: one single-thread step of the 201M "
                                                      "particles takes over a minute; c3_1t is the single-thread rate"}
    return out


def run_reference(args):
    """--impl reference: the reference's own CPU implementation, rank 0 only,
    on the same workload and metric as our arm: each benchmark step is one
    PIC step of the workload's 64x32x32-cell periodic sample (REF_SAMPLE_CELLS)
    on all host cores."""
    configs = importlib.import_module("0buf_b200.configs")
    cfg = workload_cfg(args, configs)
    if not uniform(cfg):
        return {"impl": "reference", "unavailable": NONUNIFORM_NOTE}
    threads = cpu_threads()
    kind = ref_kind()
    sim = cpu_sim(cfg, REF_SAMPLE_CELLS, threads, kind)
    n = sim.num_particles()
    for _ in range(args.warmup):
        assert sim.step() == 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        assert sim.step() == 0
    dt = time.perf_counter() - t0
    sim.close()
    value = n * args.steps / dt
    n_full = int(cfg["cells"][0] * cfg["cells"][1] * cfg["cells"][2]) * cfg["ppc"] * 3
    sample = (f"{args.steps} steps (after {args.warmup} warm-up) of a {'x'.join(map(str, REF_SAMPLE_CELLS))}-cell periodic "
              f"sub-box of the workload at its density ({n:,} particles), {threads} threads; "
              f"{'reference functions compiled for the host (oracle/_ref)' if kind == 'reference' else 'C restatement of the reference (oracle/cpu_pic.c)'}")
    return {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "form": "reference CPU path (FP64)",
            "config": workload_config(args, cfg, n_full, 1),
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def workload_cfg(args, configs):
    cfg = dict(configs.CONFIGS[args.config])
    if args.cells:
        cfg["cells"] = tuple(int(c) for c in args.cells.split(","))
    if args.ppc:
        cfg["ppc"] = args.ppc
    return cfg


def workload_config(args, cfg, n_per_gpu, world):
    """The `config` object of both arms: the workload, nothing of the arm."""
    cells = cfg["cells"]
    name = args.config if not (args.cells or args.ppc) else "custom"
    return {"workload": f"{name}: {cells[0]}x{cells[1]}x{cells[2]} cells, {cfg['ppc']} particles/cell/species x 3 "
                        f"species = {n_per_gpu:,} particles per GPU",
            "cells": list(cells), "ppc": cfg["ppc"], "species": 3, "tau": cfg["tau"], "h": cfg["h"],
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({28 * n_per_gpu / 1e9:.1f} GB of FP32-form particles; no flush needed)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="c2")
    ap.add_argument("--form", choices=["fp32", "fp64"], default=None)
    ap.add_argument("--cells", default=None, help="override cells, e.g. 128,64,64 (profiling cases)")
    ap.add_argument("--ppc", type=int, default=None, help="override particles per cell per species")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-run section")
    ap.add_argument("--adjoint-dirs", type=int, default=4,
                    help="random single-particle directions of the finite-difference check")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--stress-adjoint", action="store_true",
                    help="also run the stress configuration's differentiable run at full size (FP32, two checkpoint levels)")
    ap.add_argument("--no-fd", action="store_true",
                    help="skip the finite-difference checks of the differentiable runs (timings only)")
    ap.add_argument("--adjoint-steps", type=int, default=0,
                    help="steps of the adjoint configuration's run (default: its 300; shorter for profiling)")
    ap.add_argument("--adjoint-cells", default=None, help="override the adjoint configuration's cells (profiling)")
    ap.add_argument("--adjoint-ppc", type=int, default=0, help="override its particles per cell (profiling)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="run both forms this many steps with energies every step (FP32 error history against "
                         "FP64 from the same seed; 0 skips it)")
    ap.add_argument("--reference-inner", type=int, default=20)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    dist = Dist()
    if args.impl == "reference":
        if dist.rank != 0:
            return
        print(json.dumps(run_reference(args)), flush=True)
        return
    dist.init()
    try:
        out = run_ours(args, dist)
    finally:
        dist.barrier()
        dist.close()
    if dist.rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
