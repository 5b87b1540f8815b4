"""The benchmark configurations of the 0buf PIC step as plain data.

Normalised units: c = 1, omega_pe = 1 at density 1.  The reference's deposit
has no 1/volume (pqr, cell.h:1578-1616: the node weights of one particle sum
to its charge weight times the velocity) and the E update subtracts tau*J
(kernels.cu:1101), so omega_pe^2 = sum over a cell of q_w * (q/m).  The
reference sets the per-cell charge sum to the density (getMassCharge,
maxwell.cu:606-619), so the macro-particle charge weight is
``q_w = sign(q/m) * density / ppc``.
"""
from __future__ import annotations

import math

# config-0 species (ion, background electron, beam electron); the sort ids are
# particle_sorts (particle_types.h:11) and also the species index
SPECIES_BEAM_PLASMA = [
    dict(name="ion", sort=0, q_m=1.0 / 1836.0, density=1.01, drift=(0.0, 0.0, 0.0), vth=0.0),
    dict(name="electron", sort=1, q_m=-1.0, density=1.0, drift=(0.0, 0.0, 0.0), vth=0.02),
    dict(name="beam", sort=2, q_m=-1.0, density=0.01, drift=(0.2, 0.0, 0.0), vth=0.002),
]

CONFIGS = {
    # plain FP64 on the reference CPU path; parity case
    "c0": dict(cells=(32, 4, 4), h=0.1, tau=0.02, steps=100, ppc=32, precision="fp64"),
    # FP64 plain form at scale, ~201M particles
    "c1": dict(cells=(256, 64, 64), h=0.1, tau=0.02, steps=200, ppc=64, precision="fp64"),
    # FP32 mixed form, ~805M particles: the headline throughput case
    "c2": dict(cells=(512, 128, 128), h=0.1, tau=0.02, steps=1000, ppc=32, precision="fp32"),
    # adjoint / differentiation case
    "c3": dict(cells=(128, 32, 32), h=0.1, tau=0.02, steps=300, ppc=32, precision="fp64"),
    # stress: non-uniform electron density, hot electrons, dt = 0.05
    "c4": dict(cells=(256, 64, 64), h=0.1, tau=0.05, steps=500, ppc=64, precision="fp32", species=None),
}


# stress configuration c4: background electrons with density
# (1 + 0.5 cos(2 pi x / Lx)) x (1 + 7 exp(-d^2 / (2 (4 cells)^2))) -- a bump of
# 8x the local background at the box centre -- normalised to a mean of ppc
# particles per cell; ions with the same per-cell counts (same profile and
# count seed: neutral cell by cell up to the beam); hot electrons vth = 0.1;
# beam uniform as in c0
C4_PROFILE = dict(cos_amp=0.5, bump_peak=8.0, bump_sigma=4.0, bump_centre=(-1.0, -1.0, -1.0), count_seed=4)
SPECIES_STRESS = [
    dict(SPECIES_BEAM_PLASMA[0], profile=C4_PROFILE),
    dict(SPECIES_BEAM_PLASMA[1], vth=0.1, profile=C4_PROFILE),
    dict(SPECIES_BEAM_PLASMA[2]),
]


CONFIGS["c4"]["species"] = SPECIES_STRESS


def init_config_species(sim, cfg: dict, seed_base: int = 0):
    """Generate the species of a configuration on the device (uniform, or the
    stress profile for c4)."""
    ppc = cfg["ppc"]
    for i, s in enumerate(cfg.get("species", SPECIES_BEAM_PLASMA)):
        if "profile" in s:
            sim.init_species_profile(i, dict(s["profile"], ppc_mean=ppc), s["drift"], s["vth"], seed_base + i)
        else:
            sim.init_species(i, ppc, s["drift"], s["vth"], seed_base + i)


def charge_weight(q_m: float, density: float, ppc: int) -> float:
    """Signed macro-particle charge weight ``Particle::m`` (particle.h:43)."""
    return math.copysign(density / ppc, q_m)


def species_table(ppc: int, species=None):
    """[(q_m, m, sort)] for the C ABI."""
    species = species or SPECIES_BEAM_PLASMA
    return [(s["q_m"], charge_weight(s["q_m"], s["density"], ppc), s["sort"]) for s in species]


def box(cfg: dict):
    n = cfg["cells"]
    return tuple(float(c) * cfg["h"] for c in n)
