"""The reference's control-point checks (compare.h / compare.cxx,
service_functions.cu:180-198), applied to device state read through the C ABI.

- ``compare(a, b, tol)``: fraction of elements with |a-b| < tol (compare.cxx:9-36)
- ``comd(a, b)``: |a-b| < TOLERANCE = 1e-15 (compare.cxx:38-41, compare.h:13)
- ``check_array_silent(a, b)``: sqrt(sum (a-b)^2 / size), the absolute RMS of
  CheckArraySilent (service_functions.cu:180-198)
- ``rel_l2(a, b)``: ||a-b|| / ||b||, the parity measure of the plain form
"""
from __future__ import annotations

import numpy as np

TOLERANCE = 1e-15        # compare.h:13
SIZE_TOLERANCE = 1e-10   # compare.h:14
PARTICLE_TOLERANCE = 1e-10  # run_control.h:53


def compare(a, b, tol: float) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    if a.size == 0:
        return 0.0
    return float(np.count_nonzero(np.abs(a - b) < tol)) / a.size


def comd(a: float, b: float) -> bool:
    return abs(a - b) < TOLERANCE


def check_array_silent(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.sqrt(np.sum((a - b) ** 2) / a.size))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    if nb == 0.0:
        return 0.0 if d == 0.0 else float("inf")
    return float(d / nb)


def canonical_particles(cell, arrays):
    """Per-cell sorted particle table: rows (cell, x, y, z, px, py, pz) sorted by
    cell then by position, so two states can be compared independently of the
    order of particles inside a cell."""
    cols = [np.asarray(cell, dtype=np.float64)] + [np.asarray(a, dtype=np.float64) for a in arrays]
    tab = np.stack(cols, axis=1)
    order = np.lexsort(tuple(tab[:, c] for c in range(tab.shape[1] - 1, -1, -1)))
    return tab[order]


class ControlPointChecker:
    """Compares the device state at a control point with a reference state
    provider (a callable ``(num, nt) -> dict`` of field arrays), like
    Plasma::checkControlPoint (gpu_plasma.h:1170-1284) does against Fortran
    dumps.  Returns one row per check: RMS difference per field."""

    def __init__(self, provider, fields=("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz")):
        self.provider = provider
        self.fields = fields

    def __call__(self, plasma, num, nt):
        ref = self.provider(num, nt)
        if ref is None:
            return None
        row = dict(nt=nt, num=num)
        for f in self.fields:
            if f in ref:
                row[f] = check_array_silent(plasma.sim.get_field(f), ref[f])
        return row
