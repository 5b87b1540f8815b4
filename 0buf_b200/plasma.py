"""Host-side mirror of the reference's step driver, over the C ABI.

``PicSimulation`` is a thin owner of one ``pic_handle``.  ``Plasma`` keeps the
reference's host surface (class Plasma, gpu_plasma.h:97-2355): the same
constructor arguments as ``main.cu:14``, ``Initialize`` / ``Compute`` /
``Step`` and the sub-steps of ``Step`` with their control-point ids, so that a
user of the reference finds the same names.  All arithmetic runs in the CUDA
library; this module only moves arguments and arrays.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import _capi
from ._capi import PicConfig, PicError, dptr, iptr
from .configs import SPECIES_BEAM_PLASMA, charge_weight


class PicSimulation:
    """One PIC state on one GPU (``pic_create`` .. ``pic_destroy``)."""

    def __init__(self, cells: Sequence[int], lengths: Sequence[float], tau: float,
                 species: Sequence[tuple], precision: str = "fp64", ghosts: str = "reference",
                 device: int = 0, tile: Sequence[int] | None = None, capacity_slack: float = 0.25,
                 outbox_fraction: float = 0.04, capacity_pad: int = -1):
        self.lib = _capi.load()
        cfg = PicConfig()
        self.lib.pic_config_init(C.byref(cfg))
        cfg.nx, cfg.ny, cfg.nz = (int(c) for c in cells)
        cfg.lx, cfg.ly, cfg.lz = (float(v) for v in lengths)
        cfg.tau = float(tau)
        cfg.precision = {"fp64": _capi.PIC_FP64_PLAIN, "fp32": _capi.PIC_FP32_MIXED}[precision]
        cfg.ghosts = {"reference": _capi.PIC_GHOSTS_REFERENCE, "periodic": _capi.PIC_GHOSTS_PERIODIC}[ghosts]
        cfg.nspecies = len(species)
        for i, (q_m, m, sort) in enumerate(species):
            cfg.species[i].q_m = q_m
            cfg.species[i].m = m
            cfg.species[i].sort = sort
        cfg.device = device
        cfg.capacity_slack = capacity_slack
        cfg.outbox_fraction = outbox_fraction
        cfg.capacity_pad = capacity_pad
        if tile is not None:
            for a in range(3):
                cfg.tile[a] = int(tile[a])
        self.cfg = cfg
        self.precision = precision
        self.cells = tuple(int(c) for c in cells)
        self.shape = tuple(c + 2 for c in self.cells)
        self.nspecies = len(species)
        h = C.c_void_p()
        rc = self.lib.pic_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise PicError(rc, "pic_create")
        self.h = h

    # ------------------------------------------------------------- helpers
    def _ck(self, rc: int, where: str):
        if rc != 0:
            detail = self.lib.pic_last_error_string(self.h).decode(errors="replace") if self.h else ""
            raise PicError(rc, where, detail)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pic_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------- particles
    def load_particles(self, species: int, x, y, z, px, py, pz) -> int:
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, px, py, pz)]
        n = arrs[0].size
        ins = C.c_int64(0)
        self._ck(self.lib.pic_load_particles(self.h, species, n, *[dptr(a) for a in arrs], C.byref(ins)),
                 "pic_load_particles")
        return ins.value

    def load_particles_cells(self, species: int, cell, ox, oy, oz, px, py, pz) -> int:
        """Native 28-byte layout: reference cell number, FP32 offsets and momenta.
        Arrays may be numpy arrays or pinned host torch tensors (anything with
        a host data pointer: ``.ctypes.data`` or ``.data_ptr()``)."""
        ptrs = [_host_ptr(a) for a in (cell, ox, oy, oz, px, py, pz)]
        n = _length(cell)
        ins = C.c_int64(0)
        self._ck(self.lib.pic_load_particles_cells(self.h, species, n, *ptrs, C.byref(ins)),
                 "pic_load_particles_cells")
        return ins.value

    def get_particles_cells(self, species: int, out) -> int:
        """Exports one species into ``out`` = (cell, ox, oy, oz, px, py, pz) host arrays."""
        ptrs = [_host_ptr(a) for a in out]
        got = C.c_int64(0)
        self._ck(self.lib.pic_get_particles_cells(self.h, species, _length(out[0]), *ptrs, C.byref(got)),
                 "pic_get_particles_cells")
        return got.value

    def init_species(self, species: int, ppc: int, drift=(0.0, 0.0, 0.0), vth: float = 0.0, seed: int = 0):
        self._ck(self.lib.pic_init_species_device(self.h, species, ppc, *[float(d) for d in drift], float(vth),
                                                  int(seed)), "pic_init_species_device")

    def init_species_profile(self, species: int, profile: dict, drift=(0.0, 0.0, 0.0), vth: float = 0.0,
                             seed: int = 0):
        """Device generator with per-cell counts from a density profile
        (keys of ``pic_profile``: ppc_mean, cos_amp, bump_peak, bump_sigma,
        bump_centre, count_seed)."""
        prof = make_profile(profile)
        self._ck(self.lib.pic_init_species_profile(self.h, species, C.byref(prof), *[float(d) for d in drift],
                                                   float(vth), int(seed)), "pic_init_species_profile")

    def num_particles(self, species: int = -1) -> int:
        n = self.lib.pic_num_particles(self.h, species)
        if n < 0:
            self._ck(int(n), "pic_num_particles")
        return int(n)

    def particles(self, species: int) -> dict:
        n = self.num_particles(species)
        out = {k: np.zeros(max(n, 1)) for k in ("x", "y", "z", "px", "py", "pz")}
        cell = np.zeros(max(n, 1), np.int32)
        got = C.c_int64(0)
        self._ck(self.lib.pic_get_particles(self.h, species, max(n, 1), *[dptr(out[k]) for k in
                                            ("x", "y", "z", "px", "py", "pz")], iptr(cell), C.byref(got)),
                 "pic_get_particles")
        m = got.value
        res = {k: v[:m] for k, v in out.items()}
        res["cell"] = cell[:m]
        return res

    def cell_counts(self) -> np.ndarray:
        c = np.zeros(int(np.prod(self.shape)), np.int32)
        self._ck(self.lib.pic_get_cell_counts(self.h, iptr(c)), "pic_get_cell_counts")
        return c

    def cell_particles(self, species: int, cell: int) -> dict:
        """One interior cell's particles of one species (pic_get_cell_particles):
        x y z px py pz (global FP64) and slot in slot order, plus the tile bin's
        first slot; cell is the reference cell number."""
        n = C.c_int64(0)
        off = C.c_int64(0)
        # first call for the count (cap 0 returns PIC_ERR_ARG when the cell holds particles)
        rc = self.lib.pic_get_cell_particles(self.h, species, int(cell), 0, *([None] * 6), None, C.byref(n), C.byref(off))
        m = int(n.value)
        if rc != 0 and m == 0:
            self._ck(rc, "pic_get_cell_particles")
        out = {k: np.zeros(max(m, 1)) for k in ("x", "y", "z", "px", "py", "pz")}
        slot = np.zeros(max(m, 1), np.int64)
        self._ck(self.lib.pic_get_cell_particles(self.h, species, int(cell), m, *[dptr(out[k]) for k in
                                                 ("x", "y", "z", "px", "py", "pz")], slot.ctypes.data_as(
                                                 C.POINTER(C.c_int64)), C.byref(n), C.byref(off)),
                 "pic_get_cell_particles")
        res = {k: v[:m] for k, v in out.items()}
        res["slot"] = slot[:m]
        res["bin_offset"] = int(off.value)
        return res

    # -------------------------------------------------------------- fields
    def get_field(self, name: str) -> np.ndarray:
        a = np.zeros(int(np.prod(self.shape)))
        self._ck(self.lib.pic_get_field(self.h, _capi.FIELD_ID[name], dptr(a)), f"pic_get_field({name})")
        return a

    def set_field(self, name: str, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        assert a.size == int(np.prod(self.shape))
        self._ck(self.lib.pic_set_field(self.h, _capi.FIELD_ID[name], dptr(a)), f"pic_set_field({name})")

    def fields(self, names=_capi.FIELDS) -> dict:
        return {n: self.get_field(n) for n in names}

    # --------------------------------------------------------------- steps
    def step(self, nt: int = 0):
        self._ck(self.lib.pic_step(self.h, nt), "pic_step")

    def run(self, nsteps: int, energies: bool = False):
        if energies:
            e = np.zeros((nsteps, 4))
            self._ck(self.lib.pic_run(self.h, nsteps, dptr(e)), "pic_run")
            return e
        self._ck(self.lib.pic_run(self.h, nsteps, None), "pic_run")
        return None

    def substep(self, name: str):
        self._ck(getattr(self.lib, "pic_" + name)(self.h), "pic_" + name)

    def sync(self):
        self._ck(self.lib.pic_sync(self.h), "pic_sync")

    # --------------------------------------------------------- diagnostics
    def energy(self) -> np.ndarray:
        e = np.zeros(4)
        self._ck(self.lib.pic_energy(self.h, dptr(e)), "pic_energy")
        return e

    def charge_density(self) -> np.ndarray:
        """rho on the cell-centre nodes (linear weights, folded), reference layout."""
        a = np.zeros(int(np.prod(self.shape)))
        self._ck(self.lib.pic_charge_density(self.h, dptr(a)), "pic_charge_density")
        return a

    def gauss_residual(self) -> np.ndarray:
        """G = div E - rho on the interior nodes (0 on ghosts), reference layout."""
        a = np.zeros(int(np.prod(self.shape)))
        self._ck(self.lib.pic_gauss_residual(self.h, dptr(a)), "pic_gauss_residual")
        return a

    def dump_write(self, path: str):
        """``pic_dump_write``: checkpoint in the reference's Fortran-record dump format."""
        self._ck(self.lib.pic_dump_write(self.h, os.fsencode(path)), "pic_dump_write")

    def dump_read(self, path: str):
        """``pic_dump_read``: resume from a dump (same grid and species)."""
        self._ck(self.lib.pic_dump_read(self.h, os.fsencode(path)), "pic_dump_read")

    def momentum(self) -> np.ndarray:
        """(nspecies, 3) total mechanical momentum sum (m/q_m) p per species, FP64."""
        out = np.zeros(3 * self.nspecies)
        self._ck(self.lib.pic_momentum(self.h, dptr(out)), "pic_momentum")
        return out.reshape(self.nspecies, 3)

    def gauss_check(self, set_baseline: bool = False) -> np.ndarray:
        """[max |G - G0|, max |rho|, rms(G - G0), max |G0|]; set_baseline stores G as G0."""
        out = np.zeros(4)
        self._ck(self.lib.pic_gauss_check(self.h, int(bool(set_baseline)), dptr(out)), "pic_gauss_check")
        return out

    def energy_reference(self) -> float:
        e = np.zeros(1)
        self._ck(self.lib.pic_energy_reference(self.h, dptr(e)), "pic_energy_reference")
        return float(e[0])

    def counters(self) -> np.ndarray:
        c = np.zeros(4, np.int64)
        self.lib.pic_step_counters(self.h, c.ctypes.data_as(_capi.I64))
        return c

    def timings(self) -> np.ndarray:
        """[b_half, push kernel, migration arrivals, second field half, whole step] in ms."""
        t = np.zeros(5, np.float32)
        self.lib.pic_step_timings(self.h, t.ctypes.data_as(_capi.F))
        return t

    def layout(self) -> dict:
        v = np.zeros(4, np.int64)
        self._ck(self.lib.pic_layout_info(self.h, v.ctypes.data_as(_capi.I64)), "pic_layout_info")
        return dict(tiles=int(v[0]), slots=int(v[1]), bytes_per_particle=int(v[2]), nodes=int(v[3]))

    # ------------------------------------------------- differentiable run
    def forward(self, steps: int, ckpt_every: int, sub_every: int | None = None):
        """``pic_forward``: advance ``steps`` steps, checkpointing every ``ckpt_every``
        (``pic_forward2`` with a second checkpoint level every ``sub_every`` steps)."""
        if sub_every is None:
            self._ck(self.lib.pic_forward(self.h, int(steps), int(ckpt_every)), "pic_forward")
        else:
            self._ck(self.lib.pic_forward2(self.h, int(steps), int(ckpt_every), int(sub_every)), "pic_forward2")
        self._fwd_steps = int(steps)

    def branch_record(self, on: bool = True):
        """``pic_branch_record``: the next forward (FP64) records its discrete choices."""
        self._ck(self.lib.pic_branch_record(self.h, int(bool(on))), "pic_branch_record")

    def forward_replay(self, steps: int, recorded: "PicSimulation"):
        """``pic_forward_replay``: forward that replays ``recorded``'s choices (frozen branches)."""
        self._ck(self.lib.pic_forward_replay(self.h, int(steps), recorded.h), "pic_forward_replay")
        self._fwd_steps = int(steps)

    def perturb_momenta(self, species: int, dp: np.ndarray, eps: float):
        """``pic_perturb_momenta``: p += eps * dp, dp (n, 3) in ``particles(species)`` order."""
        a = np.ascontiguousarray(dp, dtype=np.float64).reshape(-1, 3)
        self._ck(self.lib.pic_perturb_momenta(self.h, species, a.shape[0], dptr(a), float(eps)), "pic_perturb_momenta")

    def history(self) -> np.ndarray:
        """(steps, 3): h^3 * sum over nodes 1..N of E_c^2 after each step of the last forward run."""
        out = np.zeros((self._fwd_steps, 3))
        self._ck(self.lib.pic_forward_history(self.h, dptr(out)), "pic_forward_history")
        return out

    @staticmethod
    def make_loss(field: str = "Ex", window: int = 1, species: int = 0, drift=(0.0, 0.0, 0.0),
                  vth: float = 0.0) -> _capi.PicLoss:
        L = _capi.PicLoss()
        L.field = {"Ex": 0, "Ey": 1, "Ez": 2}[field]
        L.window = int(window)
        L.species = int(species)
        for a in range(3):
            L.drift[a] = float(drift[a])
        L.vth = float(vth)
        return L

    def loss_value(self, **loss) -> float:
        v = np.zeros(1)
        L = self.make_loss(**loss)
        self._ck(self.lib.pic_loss_value(self.h, C.byref(L), dptr(v)), "pic_loss_value")
        return float(v[0])

    def backward(self, want_p0: bool = True, **loss) -> dict:
        """``pic_backward``: loss value, dL/d drift, dL/d vth and dL/dp0 (n, 3) of ``species``,
        in ``particles(species)`` order as of the call to ``forward``."""
        L = self.make_loss(**loss)
        G = _capi.PicGrads()
        buf = None
        if want_p0:
            n = self.num_particles(L.species)  # the differentiable run keeps every particle
            buf = np.zeros((max(n, 1), 3))
            G.n = n
            G.d_p0 = buf.ctypes.data
        self._ck(self.lib.pic_backward(self.h, C.byref(L), C.byref(G)), "pic_backward")
        out = dict(loss=G.loss, d_drift=np.array(G.d_drift[:]), d_vth=G.d_vth, n=int(G.n))
        if buf is not None:
            out["d_p0"] = buf[:G.n]
        return out

    def adjoint_timings(self) -> np.ndarray:
        """[forward, backward] device milliseconds of the last differentiable run."""
        t = np.zeros(2, np.float32)
        self._ck(self.lib.pic_adjoint_timings(self.h, t.ctypes.data_as(_capi.F)), "pic_adjoint_timings")
        return t

    def adjoint_free(self):
        self._ck(self.lib.pic_adjoint_free(self.h), "pic_adjoint_free")


def _host_ptr(a):
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())  # torch tensor on the host


def _length(a) -> int:
    return int(a.size if isinstance(a, np.ndarray) else a.numel())


FIELD_ORDER = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz")
_PKEYS = ("x", "y", "z", "px", "py", "pz")


def mumu_name(num: int, nt: int) -> str:
    """The reference's dump file name ``mumu%03d%08d.dat`` (``pic_mumu_name``)."""
    buf = C.create_string_buffer(64)
    rc = _capi.load().pic_mumu_name(int(num), int(nt), buf, 64)
    if rc != 0:
        raise PicError(rc, "pic_mumu_name")
    return buf.value.decode()


def mumu_write(path: str, cells, fields=None, sorts=()):
    """``pic_mumu_write``: fields = dict name -> (Nx+2)(Ny+2)(Nz+2) array (missing: zeros);
    sorts = [dict(q_m, m, x, y, z, px, py, pz)]."""
    d = _capi.PicMumu()
    d.nx, d.ny, d.nz = (int(c) for c in cells)
    keep = []
    for a, name in enumerate(FIELD_ORDER):
        if fields is not None and name in fields:
            arr = np.ascontiguousarray(fields[name], dtype=np.float64).ravel()
            keep.append(arr)
            d.fields[a] = arr.ctypes.data
    d.nsort = len(sorts)
    for s, sp in enumerate(sorts):
        d.q_m[s] = float(sp["q_m"])
        d.m[s] = float(sp["m"])
        n = None
        for a, k in enumerate(_PKEYS):
            arr = np.ascontiguousarray(sp[k], dtype=np.float64).ravel()
            n = arr.size if n is None else n
            assert arr.size == n
            keep.append(arr)
            d.p[s][a] = arr.ctypes.data
        d.count[s] = n or 0
    rc = _capi.load().pic_mumu_write(os.fsencode(path), C.byref(d))
    if rc != 0:
        raise PicError(rc, "pic_mumu_write")


def mumu_read(path: str, cells):
    """``pic_mumu_read``: (fields dict, [dict(q_m, m, x, y, z, px, py, pz)])."""
    lib = _capi.load()
    d = _capi.PicMumu()
    d.nx, d.ny, d.nz = (int(c) for c in cells)
    rc = lib.pic_mumu_read_counts(os.fsencode(path), C.byref(d))
    if rc != 0:
        raise PicError(rc, "pic_mumu_read_counts")
    nodes = int(np.prod([c + 2 for c in cells]))
    fields = {name: np.zeros(nodes) for name in FIELD_ORDER}
    for a, name in enumerate(FIELD_ORDER):
        d.fields[a] = fields[name].ctypes.data
    sorts = []
    for s in range(d.nsort):
        sp = {k: np.zeros(int(d.count[s])) for k in _PKEYS}
        for a, k in enumerate(_PKEYS):
            d.p[s][a] = sp[k].ctypes.data if sp[k].size else None
        sorts.append(sp)
    rc = lib.pic_mumu_read(os.fsencode(path), C.byref(d))
    if rc != 0:
        raise PicError(rc, "pic_mumu_read")
    for s, sp in enumerate(sorts):
        sp["q_m"], sp["m"] = float(d.q_m[s]), float(d.m[s])
    return fields, sorts


def make_profile(profile: dict):
    p = _capi.PicProfile()
    p.ppc_mean = float(profile["ppc_mean"])
    p.cos_amp = float(profile.get("cos_amp", 0.0))
    p.bump_peak = float(profile.get("bump_peak", 1.0))
    p.bump_sigma = float(profile.get("bump_sigma", 0.0))
    for a, v in enumerate(profile.get("bump_centre", (-1.0, -1.0, -1.0))):
        p.bump_centre[a] = float(v)
    p.count_seed = int(profile.get("count_seed", 0))
    return p


def profile_counts(cells, profile: dict) -> np.ndarray:
    """Particles per cell of a density profile (``pic_profile_counts``), shape cells."""
    lib = _capi.load()
    counts = np.zeros(int(np.prod(cells)), np.int32)
    total = C.c_int64(0)
    prof = make_profile(profile)
    rc = lib.pic_profile_counts(int(cells[0]), int(cells[1]), int(cells[2]), C.byref(prof),
                                counts.ctypes.data_as(_capi.I32), C.byref(total))
    if rc != 0:
        raise PicError(rc, "pic_profile_counts")
    return counts.reshape(tuple(int(c) for c in cells))


def host_species(cells, lengths, species_index: int, ppc: int, drift=(0.0, 0.0, 0.0), vth: float = 0.0,
                 seed: int = 0):
    """The seeded generator on the host (``pic_init_species_host``): x, y, z, px, py, pz arrays."""
    lib = _capi.load()
    n = int(np.prod(cells)) * ppc
    arrs = [np.zeros(n) for _ in range(6)]
    rc = lib.pic_init_species_host(int(cells[0]), int(cells[1]), int(cells[2]), *[float(v) for v in lengths],
                                   species_index, ppc, *[float(d) for d in drift], float(vth), int(seed),
                                   *[dptr(a) for a in arrs])
    if rc != 0:
        raise PicError(rc, "pic_init_species_host")
    return arrs


class Rnd:
    """The reference's random numbers (``rnd_uniform`` / ``rnd_gaussian``,
    maxwell.cu:187-197) with the state held here: ``Rnd()`` starts where the
    reference starts, ``Rnd(ix, iy, iz, store)`` anywhere else."""

    def __init__(self, ix=None, iy=None, iz=None, store=None):
        self._lib = _capi.load()
        self.state = _capi.PicRnd()
        self._lib.pic_rnd_init(C.byref(self.state))
        for k, v in (("ix", ix), ("iy", iy), ("iz", iz), ("store", store)):
            if v is not None:
                setattr(self.state, k, v)

    def uniform(self, n: int | None = None):
        if n is None:
            return self._lib.pic_rnd_uniform(C.byref(self.state))
        return np.array([self._lib.pic_rnd_uniform(C.byref(self.state)) for _ in range(int(n))])

    def gaussian(self, mean=0.0, sd=1.0, n: int | None = None):
        if n is None:
            return self._lib.pic_rnd_gaussian(C.byref(self.state), float(mean), float(sd))
        return np.array([self._lib.pic_rnd_gaussian(C.byref(self.state), float(mean), float(sd))
                         for _ in range(int(n))])

    @staticmethod
    def table() -> np.ndarray:
        out = np.zeros(41)
        rc = _capi.load().pic_rnd_table(dptr(out))
        if rc != 0:
            raise PicError(rc, "pic_rnd_table")
        return out


QUIET_SORTS = ("ions", "electrons", "beam")


def quiet_params(**overrides) -> _capi.PicQuiet:
    """The reference's quiet-start parameters (``pic_quiet_defaults``) with overrides."""
    q = _capi.PicQuiet()
    rc = _capi.load().pic_quiet_defaults(C.byref(q))
    if rc != 0:
        raise PicError(rc, "pic_quiet_defaults")
    for k, v in overrides.items():
        if not hasattr(q, k):
            raise KeyError(k)
        setattr(q, k, v)
    return q


def quiet_start(**overrides):
    """The reference's quiet start (``pic_quiet_start``; getUniformMaxwellianParticles,
    maxwell.cu:676-757): dict of ions / electrons / beam, each a dict of x y z
    px py pz arrays plus q_m and m (getMassCharge).  Keyword arguments
    override the reference's parameters (n_ions, lx, beam_ly, ...)."""
    q = quiet_params(**overrides)
    n = int(q.n_ions)
    if n < 0:
        raise PicError(-1, "pic_quiet_start: n_ions < 0")
    sizes = (n, 2 * n, n)
    arrs = [[np.zeros(sz) for _ in range(6)] for sz in sizes]
    ptrs = [(C.c_void_p * 6)(*[a.ctypes.data if a.size else None for a in group]) for group in arrs]
    nb = C.c_int64(0)
    q_m, m = np.zeros(3), np.zeros(3)
    rc = _capi.load().pic_quiet_start(C.byref(q), *ptrs, C.byref(nb), dptr(q_m), dptr(m))
    if rc != 0:
        raise PicError(rc, "pic_quiet_start")
    out = {}
    for s, (name, group) in enumerate(zip(QUIET_SORTS, arrs)):
        keep = int(nb.value) if name == "beam" else group[0].size
        out[name] = {k: a[:keep] for k, a in zip(_PKEYS, group)}
        out[name].update(q_m=float(q_m[s]), m=float(m[s]))
    return out


class Plasma:
    """Mirror of the reference's ``class Plasma`` (gpu_plasma.h:97).

    ``Plasma(Nx, Ny, Nz, Lx, Ly, Lz, ni, n_per_cell, ion_q_m, tau)`` takes the
    arguments of the reference constructor (gpu_plasma.h:1574-1589, called as
    in main.cu:14).  ``Initialize`` loads the beam-plasma species of the
    benchmark configurations (ions of q/m = ion_q_m and density 1.01*ni,
    electrons of density ni, beam of density 0.01*ni) with ``n_per_cell``
    particles per cell per species from a seeded generator; with
    ``loader="quiet_start"`` it loads the reference's own initial state
    instead (InitializeCPU, init.cu:111-139: getUniformMaxwellianParticles,
    maxwell.cu:676-757, whose parameters -- 1.6M ions, lp = 1000, the box of
    main.cu:14 -- are its own, overridable through ``quiet``), with the charge
    weights of getMassCharge (maxwell.cu:598-612).
    """

    TOTAL_STEPS = 5  # run_control.h:10

    def __init__(self, Nx, Ny, Nz, Lx, Ly, Lz, ni, n_per_cell, ion_q_m, tau, precision="fp64",
                 ghosts="reference", device=0, seed=0, species=None, loader="generator", quiet=None):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.ni, self.n_per_cell, self.ion_q_m, self.tau = ni, n_per_cell, ion_q_m, tau
        self.seed = seed
        if loader not in ("generator", "quiet_start"):
            raise ValueError(loader)
        self.loader, self.quiet = loader, dict(quiet or {})
        if loader == "quiet_start":
            w = quiet_start(**dict(self.quiet, n_ions=0))
            table = [(w[k]["q_m"], w[k]["m"], sort) for sort, k in enumerate(QUIET_SORTS)]
            self.species = [dict(name=k, sort=sort, q_m=w[k]["q_m"], m=w[k]["m"]) for sort, k in enumerate(QUIET_SORTS)]
        else:
            if species is None:
                species = [dict(s) for s in SPECIES_BEAM_PLASMA]
                species[0]["q_m"] = ion_q_m
                for s in species:
                    s["density"] = s["density"] * ni
            self.species = species
            table = [(s["q_m"], charge_weight(s["q_m"], s["density"], n_per_cell), s["sort"]) for s in species]
        self.sim = PicSimulation((Nx, Ny, Nz), (Lx, Ly, Lz), tau, table, precision=precision, ghosts=ghosts,
                                 device=device)
        self.energy_history = []
        self.control_points = []

    # Initialize, init.cu:141-152
    def Initialize(self, host_generator: bool = False):
        if self.loader == "quiet_start":
            parts = quiet_start(**self.quiet)
            for i, k in enumerate(QUIET_SORTS):
                self.sim.load_particles(i, *[parts[k][a] for a in _PKEYS])
            return
        for i, s in enumerate(self.species):
            if host_generator:
                arrs = host_species((self.Nx, self.Ny, self.Nz), (self.Lx, self.Ly, self.Lz), i, self.n_per_cell,
                                    s["drift"], s["vth"], self.seed)
                self.sim.load_particles(i, *arrs)
            else:
                self.sim.init_species(i, self.n_per_cell, s["drift"], s["vth"], self.seed)

    # ComputeField_FirstHalfStep, gpu_plasma.h:367-397 (control point 50)
    def ComputeField_FirstHalfStep(self, nt):
        self.sim.substep("b_half")
        self.checkControlPoint(50, nt)
        self.sim.substep("stage_fields")

    # PushParticles, gpu_plasma.h:554-570 (control point 270)
    def PushParticles(self, nt):
        self.sim.substep("push_deposit")
        self.sim.substep("migrate")
        self.checkControlPoint(270, nt)

    # ComputeField_SecondHalfStep, gpu_plasma.h:399-414 (control points 275, 400, 500, 550, 600)
    def ComputeField_SecondHalfStep(self, nt):
        self.checkControlPoint(275, nt)
        self.sim.substep("j_fold")
        self.checkControlPoint(400, nt)
        self.sim.substep("b_complete")
        self.checkControlPoint(500, nt)
        self.sim.substep("e_update")
        self.checkControlPoint(550, nt)
        self.sim.substep("e_ghosts")
        self.checkControlPoint(600, nt)

    # Step, gpu_plasma.h:605-620 (the MPI sum of J is not part of the one-GPU step)
    def Step(self, nt):
        self.ComputeField_FirstHalfStep(nt)
        self.PushParticles(nt)
        self.ComputeField_SecondHalfStep(nt)
        self.Diagnose(nt)

    # Compute, gpu_plasma.h:2329-2352
    def Compute(self, total_steps=None):
        for nt in range(1, (total_steps or self.TOTAL_STEPS) + 1):
            self.Step(nt)

    # getElectricEnergy / Diagnose, gpu_plasma.h:621-686
    def getElectricEnergy(self) -> float:
        return self.sim.energy_reference()

    def Diagnose(self, nt):
        self.energy_history.append((nt, self.getElectricEnergy()))

    # checkControlPoint, gpu_plasma.h:1170-1284: a hook, see compare.ControlPointChecker
    checker = None

    def checkControlPoint(self, num, nt):
        if self.checker is not None:
            self.control_points.append(self.checker(self, num, nt))
