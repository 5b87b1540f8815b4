"""Generates the golden fixtures of the 0buf PIC step from the REFERENCE'S OWN
functions (cell.h / particle.h / kernels.cu compiled for the host by
oracle/build_ref.sh and replayed by oracle/ref_driver.cu).

Run in a container that has the reference sources:
    python tests/golden/make_golden.py
Writes tests/golden/ref_small.npz and tests/golden/ref_c0.npz, whose inputs
come from the product's host generator (pic_init_species_host, seeded) and are
stored in the fixture (small case) or pinned by a digest (c0 case) so the
fixtures stand alone; and tests/golden/ref_quiet.npz, the reference's own
default run (main.cu:14: 100x4x4 cells, box 1.1424 x 0.05 x 0.05, tau 0.001)
from the reference's own initial state (getUniformMaxwellianParticles,
maxwell.cu:676-757, pinned by a digest); and tests/golden/ref_stress.npz, the
stress configuration's profile and hot electrons (c4's species, dt 0.05) on
16x8x8 cells, inputs from the host generator thinned to the profile and
pinned by a digest.
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
pkg = importlib.import_module("0buf_b200")
from oracle import RefSim, FIELDS, SUBSTEPS  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    if a.dtype == np.float64:
        a = np.where(a == 0.0, 0.0, a)  # -0.0 and +0.0 hash alike
    return hashlib.sha256(a.tobytes()).hexdigest()


def species_inputs(cells, lengths, ppc, seed):
    out = []
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], seed)
        m = pkg.configs.charge_weight(s["q_m"], s["density"], ppc)
        out.append((s["sort"], arrs, m, s["q_m"]))
    return out


def particle_table(p):
    return np.stack([p["cell"].astype(np.float64), p["sort"].astype(np.float64), p["x"], p["y"], p["z"], p["px"],
                     p["py"], p["pz"]], axis=1)


def make_small():
    cells, h, tau, ppc, seed, steps = (8, 4, 4), 0.1, 0.02, 3, 7, 4
    # arrays each sub-step changes (snapshotted after that sub-step of step 1)
    changed = dict(b_half=("Hx", "Hy", "Hz", "Qx", "Qy", "Qz"), write_j=("Jx", "Jy", "Jz"),
                   j_fold=("Jx", "Jy", "Jz"), b_complete=("Hx", "Hy", "Hz"), e_update=("Ex", "Ey", "Ez"),
                   e_ghosts=("Ex", "Ey", "Ez"))
    lengths = tuple(c * h for c in cells)
    sim = RefSim(cells, lengths, tau)
    inputs = species_inputs(cells, lengths, ppc, seed)
    rec = dict(cells=np.array(cells), h=h, tau=tau, ppc=ppc, seed=seed, steps=steps)
    for sort, arrs, m, q_m in inputs:
        sim.add_particles(sort, *arrs, m, q_m)
        for k, a in zip(("x", "y", "z", "px", "py", "pz"), arrs):
            rec[f"in_s{sort}_{k}"] = a
        rec[f"in_s{sort}_m"] = m
        rec[f"in_s{sort}_q_m"] = q_m
    rng = np.random.default_rng(seed)
    for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        a = rng.normal(0.0, 1e-3, sim.nodes)
        sim.set_field(f, a)
        rec[f"in_{f}"] = a
    for st in range(1, steps + 1):
        for sub in SUBSTEPS:
            rc = sim.substep(sub)
            assert rc == 0, (sub, rc)
            if st == 1 and sub in changed:
                for f in changed[sub]:
                    rec[f"sub_{sub}_{f}"] = sim.get_field(f)
            if st == 1 and sub == "migrate":
                rec["sub_migrate_particles"] = particle_table(sim.particles())
        for f in FIELDS:
            rec[f"step{st}_{f}"] = sim.get_field(f)
        rec[f"step{st}_counts"] = sim.cell_counts()
        rec[f"step{st}_energy"] = sim.energy_reference()
        if st in (1, steps):
            rec[f"step{st}_particles"] = particle_table(sim.particles())
    np.savez_compressed(os.path.join(OUT, "ref_small.npz"), **rec)


def make_c0(steps=10):
    cfg = pkg.configs.CONFIGS["c0"]
    cells, h, tau, ppc, seed = cfg["cells"], cfg["h"], cfg["tau"], cfg["ppc"], 0
    lengths = tuple(c * h for c in cells)
    sim = RefSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    inputs = species_inputs(cells, lengths, ppc, seed)
    rec = dict(cells=np.array(cells), h=h, tau=tau, ppc=ppc, seed=seed, steps=steps)
    rec["inputs_digest"] = digest(np.concatenate([a for _, arrs, _, _ in inputs for a in arrs]))
    for sort, arrs, m, q_m in inputs:
        sim.add_particles(sort, *arrs, m, q_m)
    for st in range(1, steps + 1):
        assert sim.step() == 0
        for f in FIELDS:
            rec[f"step{st}_{f}_digest"] = digest(sim.get_field(f))
        rec[f"step{st}_counts"] = sim.cell_counts()
        rec[f"step{st}_energy"] = sim.energy_reference()
        rec[f"step{st}_particles_digest"] = digest(particle_table(sim.particles()))
    for f in FIELDS:
        rec[f"final_{f}"] = sim.get_field(f)
    np.savez_compressed(os.path.join(OUT, "ref_c0.npz"), **rec)


def stress_inputs(cells, lengths, ppc, seed):
    """The stress configuration's species on a small grid: the library's host
    generator (cell-major, keyed by seed, species, cell, slot) thinned to the
    c4 density profile's per-cell counts for the profiled species (cold ions,
    hot electrons of vth 0.1), uniform for the beam."""
    counts = pkg.profile_counts(cells, dict(pkg.configs.C4_PROFILE, ppc_mean=ppc)).ravel()
    cmax = int(counts.max())
    table = pkg.configs.species_table(ppc, pkg.configs.SPECIES_STRESS)
    out = []
    for i, s in enumerate(pkg.configs.SPECIES_STRESS):
        if "profile" in s:
            arrs = pkg.host_species(cells, lengths, i, cmax, s["drift"], s["vth"], seed)
            keep = (np.arange(cmax)[None, :] < counts[:, None]).ravel()
            arrs = [a[keep] for a in arrs]
        else:
            arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], seed)
        out.append((s["sort"], arrs, table[i][1], s["q_m"]))
    return out


STRESS = dict(cells=(16, 8, 8), h=0.1, tau=0.05, ppc=8, seed=3, steps=10)


def make_stress():
    cells, h, tau, ppc, seed, steps = (STRESS[k] for k in ("cells", "h", "tau", "ppc", "seed", "steps"))
    lengths = tuple(c * h for c in cells)
    sim = RefSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    inputs = stress_inputs(cells, lengths, ppc, seed)
    rec = dict(cells=np.array(cells), h=h, tau=tau, ppc=ppc, seed=seed, steps=steps)
    rec["inputs_digest"] = digest(np.concatenate([a for _, arrs, _, _ in inputs for a in arrs]))
    for sort, arrs, m, q_m in inputs:
        sim.add_particles(sort, *arrs, m, q_m)
        rec[f"in_s{sort}_count"] = arrs[0].size
    moved = 0
    prev = sim.cell_counts()
    for st in range(1, steps + 1):
        assert sim.step() == 0
        c = sim.cell_counts()
        moved += int(np.abs(c - prev).sum())
        prev = c
        for f in FIELDS:
            rec[f"step{st}_{f}_digest"] = digest(sim.get_field(f))
        rec[f"step{st}_counts"] = c
        rec[f"step{st}_energy"] = sim.energy_reference()
        rec[f"step{st}_particles_digest"] = digest(particle_table(sim.particles()))
    rec["count_changes"] = moved
    for f in FIELDS:
        rec[f"final_{f}"] = sim.get_field(f)
    np.savez_compressed(os.path.join(OUT, "ref_stress.npz"), **rec)


def control_points_dat(path):
    """nt, num and the twelve RMS differences of the reference's
    control_points.dat line (names Ex .. Qz), plus its particle figure."""
    words = open(path).read().split()
    rec = {"cp_nt": int(words[words.index("nt") + 1]), "cp_num": int(words[words.index("num") + 1])}
    names = [n for n in FIELDS] + ["particles"]
    rec["cp_names"] = np.array(names)
    rec["cp_rms"] = np.array([float(words[words.index(n) + 1]) for n in names])
    return rec


QUIET_SAMPLE = 4999  # every 4999th row of the canonical particle table


def make_quiet(steps=10):
    import oracle
    cells, lengths, tau = (100, 4, 4), (1.1424, 0.05, 0.05), 0.001
    sorts = oracle.ref_quiet_default()
    sim = RefSim(cells, lengths, tau, threads=os.cpu_count() or 1)
    rec = dict(cells=np.array(cells), lengths=np.array(lengths), tau=tau, steps=steps, sample=QUIET_SAMPLE)
    rec["inputs_digest"] = digest(np.concatenate([P[:, a] for P in sorts for a in range(6)]))
    for s, P in enumerate(sorts):
        rec[f"in_s{s}_count"] = P.shape[0]
        rec[f"in_s{s}_m"], rec[f"in_s{s}_q_m"] = P[0, 6], P[0, 7]
        sim.add_particles(s, *[np.ascontiguousarray(P[:, a]) for a in range(6)], P[0, 6], P[0, 7])
    for st in range(1, steps + 1):
        assert sim.step() == 0
        rec[f"step{st}_counts"] = sim.cell_counts()
        rec[f"step{st}_energy"] = sim.energy_reference()
        if st in (1, 5, steps):
            for f in FIELDS:
                rec[f"step{st}_{f}"] = sim.get_field(f)
    # the reference's own record of its GPU run of this case against its
    # Fortran original (control_points.dat, written by checkControlPoint,
    # gpu_plasma.h:1170-1284): RMS differences at step 5, control point 600
    rec.update(control_points_dat(os.path.join(os.environ.get("REF_DIR", "/root/reference"), "control_points.dat")))
    tab = particle_table(sim.particles())
    tab = tab[np.lexsort((tab[:, 4], tab[:, 3], tab[:, 2], tab[:, 1], tab[:, 0]))]
    rec["final_rows"] = tab.shape[0]
    rec["final_particles_sample"] = tab[::QUIET_SAMPLE]
    np.savez_compressed(os.path.join(OUT, "ref_quiet.npz"), **rec)


if __name__ == "__main__":
    if not RefSim.available():
        sys.exit("oracle/_ref/libref0buf.so missing: run oracle/build_ref.sh where the reference sources exist")
    which = sys.argv[1:] or ["small", "c0", "quiet", "stress"]
    made = []
    if "small" in which:
        make_small()
        made.append("ref_small.npz")
    if "c0" in which:
        make_c0()
        made.append("ref_c0.npz")
    if "quiet" in which:
        make_quiet()
        made.append("ref_quiet.npz")
    if "stress" in which:
        make_stress()
        made.append("ref_stress.npz")
    for f in made:
        print(f, os.path.getsize(os.path.join(OUT, f)), "bytes")
