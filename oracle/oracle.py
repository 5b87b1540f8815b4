"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrappers of the two CPU implementations of the 0buf PIC step that the
tests use as checkers (never imported by the product package):

- ``OracleSim``: the C restatement ``oracle/cpu_pic.c`` (lib/libpicoracle.so)
- ``RefSim``: the reference's own functions replayed on the host
  (``oracle/ref_driver.cu`` -> _ref/libref0buf.so, built only where the
  reference sources exist)

Both expose the same methods, sub-step ids and export layout.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "libpicoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref0buf.so")

SUBSTEPS = ["b_half", "stage", "zero_j", "push", "deposit", "write_j", "migrate", "j_fold", "b_complete",
            "e_update", "e_ghosts"]
FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"]

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)


def build_oracle() -> str:
    """Compile cpu_pic.c (make) if the library is missing or stale."""
    src = os.path.join(HERE, "cpu_pic.c")
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return ORACLE_LIB


def _bind(lib, p):
    def f(name, res, args):
        fn = getattr(lib, p + name)
        fn.restype = res
        fn.argtypes = args
    f("create", C.c_void_p, [C.c_int] * 3 + [C.c_double] * 4)
    f("destroy", None, [C.c_void_p])
    f("add_particles", C.c_long, [C.c_void_p, C.c_int, C.c_long] + [D] * 6 + [C.c_double] * 2)
    f("set_field", C.c_int, [C.c_void_p, C.c_int, D])
    f("get_field", C.c_int, [C.c_void_p, C.c_int, D])
    f("substep", C.c_int, [C.c_void_p, C.c_int])
    f("step", C.c_int, [C.c_void_p])
    f("energy", C.c_double, [C.c_void_p])
    f("num_particles", C.c_long, [C.c_void_p])
    f("get_particles", C.c_long, [C.c_void_p, D, I, I, I])
    f("get_cell_counts", C.c_int, [C.c_void_p, I])


class _Sim:
    prefix = ""
    libpath = ""
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(cls.libpath):
                raise FileNotFoundError(cls.libpath)
            lib = C.CDLL(cls.libpath)
            _bind(lib, cls.prefix)
            cls._lib = lib
        return cls._lib

    def __init__(self, cells, lengths, tau, threads: int = 1):
        self.L = self.lib()
        self.cells = tuple(int(c) for c in cells)
        self.shape = tuple(c + 2 for c in self.cells)
        self.nodes = int(np.prod(self.shape))
        self.h = self._f("create")(*self.cells, *[float(v) for v in lengths], float(tau))
        if not self.h:
            raise ValueError("bad grid")
        self.set_threads(threads)

    def _f(self, name):
        return getattr(self.L, self.prefix + name)

    def set_threads(self, n):
        pass

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_particles(self, sort, x, y, z, px, py, pz, m, q_m) -> int:
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, px, py, pz)]
        return int(self._f("add_particles")(self.h, sort, arrs[0].size, *[a.ctypes.data_as(D) for a in arrs],
                                            float(m), float(q_m)))

    def set_field(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        assert a.size == self.nodes
        assert self._f("set_field")(self.h, FIELDS.index(name), a.ctypes.data_as(D)) == 0

    def get_field(self, name):
        a = np.zeros(self.nodes)
        assert self._f("get_field")(self.h, FIELDS.index(name), a.ctypes.data_as(D)) == 0
        return a

    def fields(self, names=FIELDS):
        return {n: self.get_field(n) for n in names}

    def substep(self, name) -> int:
        return int(self._f("substep")(self.h, SUBSTEPS.index(name)))

    def step(self) -> int:
        return int(self._f("step")(self.h))

    def energy_reference(self) -> float:
        return float(self._f("energy")(self.h))

    def num_particles(self) -> int:
        return int(self._f("num_particles")(self.h))

    def cell_counts(self):
        c = np.zeros(self.nodes, np.int32)
        self._f("get_cell_counts")(self.h, c.ctypes.data_as(I))
        return c

    def particles(self):
        """All particles in cell order then list order: dict of x y z px py pz m q_m x1 y1 z1, cell, sort, dir."""
        n = self.num_particles()
        P = np.zeros((max(n, 1), 11))
        cell = np.zeros(max(n, 1), np.int32)
        sort = np.zeros(max(n, 1), np.int32)
        d = np.zeros(max(n, 1), np.int32)
        self._f("get_particles")(self.h, P.ctypes.data_as(D), cell.ctypes.data_as(I), sort.ctypes.data_as(I),
                                 d.ctypes.data_as(I))
        keys = ["x", "y", "z", "px", "py", "pz", "m", "q_m", "x1", "y1", "z1"]
        out = {k: P[:n, i].copy() for i, k in enumerate(keys)}
        out.update(cell=cell[:n].copy(), sort=sort[:n].copy(), dir=d[:n].copy())
        return out


class OracleSim(_Sim):
    """The C restatement (oracle/cpu_pic.c)."""
    prefix = "op_"
    libpath = ORACLE_LIB

    @classmethod
    def lib(cls):
        if cls._lib is None:
            build_oracle()
            lib = super().lib()
            lib.op_set_threads.argtypes = [C.c_void_p, C.c_int]
            lib.op_energies.argtypes = [C.c_void_p, D]
            lib.op_energies.restype = C.c_int
            lib.op_status.argtypes = [C.c_void_p]
            lib.op_status.restype = C.c_int
            lib.op_gen_species.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [C.c_int, C.c_int] + \
                [C.c_double] * 4 + [C.c_uint64, C.c_int] + [D] * 6
            lib.op_gen_species.restype = C.c_int
            lib.op_init_species.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int] + [C.c_double] * 4 + \
                [C.c_uint64, C.c_double, C.c_double]
            lib.op_init_species.restype = C.c_long
        return cls._lib

    def init_species(self, sort, species_index, ppc, drift, vth, seed, m, q_m) -> int:
        """The seeded generator (gen_species) straight into the cell lists, in
        parallel over cells: the same state as add_particles of its arrays."""
        n = int(self.L.op_init_species(self.h, int(sort), int(species_index), int(ppc),
                                       *[float(d) for d in drift], float(vth), int(seed), float(m), float(q_m)))
        if n < 0:
            raise MemoryError("op_init_species")
        return n

    def set_threads(self, n):
        self.L.op_set_threads(self.h, int(n))

    def energies(self):
        e = np.zeros(4)
        self.L.op_energies(self.h, e.ctypes.data_as(D))
        return e


class RefSim(_Sim):
    """The reference's own functions replayed on the host (oracle/ref_driver.cu)."""
    prefix = "ref_"
    libpath = REF_LIB

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = super().lib()
            lib.ref_set_threads.argtypes = [C.c_int]
        return cls._lib

    def set_threads(self, n):
        self.L.ref_set_threads(int(n))

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.libpath)


def gen_species(cells, lengths, species_index, ppc, drift=(0.0, 0.0, 0.0), vth=0.0, seed=0, threads=1):
    """The library's seeded initial particles restated in C (op_gen_species):
    x, y, z, px, py, pz arrays in cell-major order, bit-identical to the
    library's pic_init_species_host."""
    lib = OracleSim.lib()
    n = int(np.prod(cells)) * int(ppc)
    arrs = [np.zeros(n) for _ in range(6)]
    rc = lib.op_gen_species(*[int(c) for c in cells], *[float(v) for v in lengths], int(species_index), int(ppc),
                            *[float(d) for d in drift], float(vth), int(seed), int(threads),
                            *[a.ctypes.data_as(D) for a in arrs])
    if rc != 0:
        raise ValueError("op_gen_species")
    return arrs


# ---------------------------------------------------------------------------
# Charge conservation (no counterpart in the reference, which has no charge
# density).  The zigzag deposit puts its nodes at cell centres: pqr
# (cell.h:1511-1693) weights node index iv of a particle's 5-node stencil by
# its distance to iv - 2.5 cells from the cell origin, so array node N sits at
# (N - 1/2) h per axis.  With rho assigned by the same linear weights and
# folded like the current (periodicCurrentElement, kernels.cu:1124-1146), and
# the E update's backward-difference divergence (emeElement,
# kernels.cu:1091-1102), G = div E - rho on the interior nodes is constant.

def charge_density(x, y, z, m, cells, h):
    """rho on the (nx+2)(ny+2)(nz+2) nodes, reference layout (flat); x, y, z
    global positions, m the signed charge weight per particle (array or
    scalar), h the cell sizes (3,)."""
    cells = tuple(int(c) for c in cells)
    shape = tuple(c + 2 for c in cells)
    r = np.zeros(shape)
    xc = np.stack([np.asarray(x) / h[0], np.asarray(y) / h[1], np.asarray(z) / h[2]], 1)
    cell = np.floor(xc).astype(np.int64)
    f = xc - cell
    up = (f >= 0.5).astype(np.int64)
    N0 = cell + up
    w1 = f + 0.5 - up
    m = np.broadcast_to(np.asarray(m, dtype=np.float64), (xc.shape[0],))
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                w = (w1[:, 0] if a else 1 - w1[:, 0]) * (w1[:, 1] if b else 1 - w1[:, 1]) * \
                    (w1[:, 2] if c else 1 - w1[:, 2])
                np.add.at(r, (N0[:, 0] + a, N0[:, 1] + b, N0[:, 2] + c), m * w)
    for ax in range(3):
        n = cells[ax]
        r = np.moveaxis(r, ax, 0)
        r[n] += r[0]
        r[1] += r[n + 1]
        r[0] = r[n]
        r[n + 1] = r[1]
        r = np.moveaxis(r, 0, ax)
    return r.ravel()


def gauss_residual(Ex, Ey, Ez, rho, cells, h):
    """G = div E - rho on the interior nodes (backward differences), 0 on the
    ghost nodes; flat reference layout."""
    cells = tuple(int(c) for c in cells)
    shape = tuple(c + 2 for c in cells)
    E = [np.asarray(a, dtype=np.float64).reshape(shape) for a in (Ex, Ey, Ez)]
    r = np.asarray(rho, dtype=np.float64).reshape(shape)
    nx, ny, nz = cells
    I, J, K = slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1)
    G = np.zeros(shape)
    G[I, J, K] = ((E[0][I, J, K] - E[0][0:nx, J, K]) / h[0] + (E[1][I, J, K] - E[1][I, 0:ny, K]) / h[1] +
                  (E[2][I, J, K] - E[2][I, J, 0:nz]) / h[2] - r[I, J, K])
    return G.ravel()


# ---------------------------------------------------------------------------
# The reference's Fortran-record dump (LoadParticleData, load_data.cu:308-341;
# readFortranBinaryArray, load_data.cu:35-63), restated with numpy, and the
# reference's own reader from the replay library.

def write_mumu_np(path, cells, fields, sorts):
    """fields: 12 arrays (Ex..Qz, reference layout); sorts: [(q_m, m, x, y, z, px, py, pz)]."""
    def rec(f, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        t = np.array([a.nbytes], dtype=np.int32).tobytes()
        f.write(t + a.tobytes() + t)
    with open(path, "wb") as f:
        for a in fields:
            rec(f, a)
        for q_m, m, *arrs in sorts:
            rec(f, np.array([len(arrs[0]), q_m, m], dtype=np.float64))
            for a in arrs:
                rec(f, a)


def read_mumu_np(path, cells):
    nodes = int(np.prod([c + 2 for c in cells]))
    raw = open(path, "rb").read()
    pos = 0

    def rec():
        nonlocal pos
        t = int(np.frombuffer(raw, np.int32, 1, pos)[0])
        a = np.frombuffer(raw, np.float64, t // 8, pos + 4).copy()
        assert int(np.frombuffer(raw, np.int32, 1, pos + 4 + t)[0]) == t
        pos += t + 8
        return a
    fields = [rec() for _ in range(12)]
    assert all(f.size == nodes for f in fields)
    sorts = []
    while pos < len(raw):
        head = rec()
        sorts.append((head[1], head[2], *[rec() for _ in range(6)]))
    return fields, sorts


def ref_read_mumu(workdir, nt, cells):
    """The reference's LoadParticleData on mumu000<nt>.dat in workdir (replay
    library only): [(x, y, z, pu, pv, pw, m, q_m) array per sort] for ion,
    electron, beam."""
    lib = RefSim.lib()
    lib.ref_mumu_load.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_long)]
    lib.ref_mumu_load.restype = C.c_int
    lib.ref_mumu_particles.argtypes = [C.c_int, D]
    lib.ref_mumu_particles.restype = C.c_long
    counts = (C.c_long * 3)()
    cwd = os.getcwd()
    try:
        os.chdir(workdir)
        rc = lib.ref_mumu_load(int(nt), *[int(c) for c in cells], counts)
    finally:
        os.chdir(cwd)
    if rc != 0:
        raise RuntimeError(f"LoadParticleData returned {rc}")
    out = []
    for s in range(3):
        a = np.zeros((max(int(counts[s]), 1), 8))
        n = lib.ref_mumu_particles(s, a.ctypes.data_as(D))
        out.append(a[:n])
    return out


# ---------------------------------------------------------------------------
# The reference's quiet start and random numbers (replay library only): the
# generator state lives in maxwell.cu's globals, which ref_rnd_* reset / set.

def _ref_rnd_lib():
    lib = RefSim.lib()
    lib.ref_rnd_set.argtypes = [C.c_long] * 3 + [C.c_double]
    lib.ref_rnd_set.restype = None
    lib.ref_rnd_reset.restype = None
    lib.ref_rnd_uniforms.argtypes = [C.c_long, D]
    lib.ref_rnd_uniforms.restype = None
    lib.ref_rnd_gaussians.argtypes = [C.c_long, C.c_double, C.c_double, D]
    lib.ref_rnd_gaussians.restype = None
    lib.ref_quiet_init.argtypes = [C.c_int, C.c_int, D, C.c_int, D, D, D]
    lib.ref_quiet_init.restype = C.c_long
    lib.ref_quiet_default.argtypes = [C.POINTER(C.c_long)]
    lib.ref_quiet_default.restype = C.c_int
    lib.ref_mumu_particles.argtypes = [C.c_int, D]
    lib.ref_mumu_particles.restype = C.c_long
    return lib


def ref_rnd(n, state=None, gaussian=None):
    """n numbers of the reference's rnd_uniform (gaussian None) or
    rnd_gaussian(mean, sd) (gaussian = (mean, sd)) from state (ix, iy, iz,
    store), default the reference's initial state (maxwell.cu:46-52)."""
    lib = _ref_rnd_lib()
    if state is None:
        lib.ref_rnd_reset()
    else:
        lib.ref_rnd_set(*[int(v) for v in state[:3]], float(state[3]))
    out = np.zeros(int(n))
    if gaussian is None:
        lib.ref_rnd_uniforms(int(n), out.ctypes.data_as(D))
    else:
        lib.ref_rnd_gaussians(int(n), float(gaussian[0]), float(gaussian[1]), out.ctypes.data_as(D))
    return out


QUIET_PAR = ("tex0", "tey0", "tez0", "beam_lx", "beam_ly", "beam_lz", "lx", "ly", "lz", "Tb", "rimp", "rbd")


def ref_quiet_init(jmb, beamf=1, meh=0, **par):
    """The reference's InitUniformMaxwellianParticles (maxwell.cu:379-536)
    from the initial generator state: (ion (6, jmb), electrons (6, 2 jmb),
    beam (6, count)) as x y z px py pz rows."""
    lib = _ref_rnd_lib()
    p = np.array([float(par[k]) for k in QUIET_PAR])
    ion, el, beam = np.zeros(6 * jmb), np.zeros(12 * jmb), np.zeros(6 * jmb)
    nb = lib.ref_quiet_init(int(beamf), int(jmb), p.ctypes.data_as(D), int(meh), ion.ctypes.data_as(D),
                            el.ctypes.data_as(D), beam.ctypes.data_as(D))
    return ion.reshape(6, jmb), el.reshape(6, 2 * jmb), beam.reshape(6, jmb)[:, :nb]


def ref_quiet_default():
    """The reference's getUniformMaxwellianParticles (maxwell.cu:676-757):
    [(n, 8) array of x y z pu pv pw m q_m] for ions, electrons, beam."""
    lib = _ref_rnd_lib()
    counts = (C.c_long * 3)()
    rc = lib.ref_quiet_default(counts)
    if rc != 0:
        raise RuntimeError(f"getUniformMaxwellianParticles returned {rc}")
    out = []
    for s in range(3):
        a = np.zeros((max(int(counts[s]), 1), 8))
        n = lib.ref_mumu_particles(s, a.ctypes.data_as(D))
        out.append(a[:n])
    return out
