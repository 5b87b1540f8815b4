"""ctypes binding of the C ABI in ``include/pic0buf.h`` (``lib/libpic0buf.so``).

Only plain pointers and sizes cross the boundary; numpy arrays are passed by
their data pointer.  The library must exist: there is no CPU fallback, and a
missing or unloadable library raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpic0buf.so")

PIC_FP64_PLAIN = 0
PIC_FP32_MIXED = 1
PIC_GHOSTS_REFERENCE = 0
PIC_GHOSTS_PERIODIC = 1
PIC_MAX_SPECIES = 8
FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}

PIC_ERR = {
    -1: "PIC_ERR_ARG", -2: "PIC_ERR_NOMEM", -3: "PIC_ERR_STENCIL", -4: "PIC_ERR_OUTBOX", -5: "PIC_ERR_HOLES",
    -6: "PIC_ERR_NAN", -7: "PIC_ERR_STATE", -8: "PIC_ERR_NOT_BUILT", -9: "PIC_ERR_NO_DEVICE",
}


class PicSpecies(C.Structure):
    _fields_ = [("q_m", C.c_double), ("m", C.c_double), ("sort", C.c_int), ("pad_", C.c_int)]


class PicConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("tau", C.c_double),
        ("precision", C.c_int), ("ghosts", C.c_int), ("nspecies", C.c_int), ("device", C.c_int),
        ("species", PicSpecies * PIC_MAX_SPECIES),
        ("capacity_slack", C.c_double), ("outbox_fraction", C.c_double),
        ("tile", C.c_int * 3),
        ("capacity_pad", C.c_int),
        ("reserved", C.c_int * 7),
    ]


class PicLoss(C.Structure):
    _fields_ = [("field", C.c_int), ("window", C.c_int), ("species", C.c_int), ("reserved_i", C.c_int),
                ("drift", C.c_double * 3), ("vth", C.c_double), ("reserved", C.c_double * 4)]


class PicGrads(C.Structure):
    _fields_ = [("loss", C.c_double), ("d_drift", C.c_double * 3), ("d_vth", C.c_double), ("n", C.c_int64),
                ("d_p0", C.c_void_p), ("reserved", C.c_double * 4)]


class PicMumu(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nsort", C.c_int),
                ("fields", C.c_void_p * 12),
                ("count", C.c_int64 * PIC_MAX_SPECIES),
                ("q_m", C.c_double * PIC_MAX_SPECIES), ("m", C.c_double * PIC_MAX_SPECIES),
                ("p", (C.c_void_p * 6) * PIC_MAX_SPECIES)]


class PicRnd(C.Structure):
    _fields_ = [("ix", C.c_int32), ("iy", C.c_int32), ("iz", C.c_int32), ("store", C.c_double)]


class PicQuiet(C.Structure):
    _fields_ = [("n_ions", C.c_int64), ("tex0", C.c_double), ("tey0", C.c_double), ("tez0", C.c_double),
                ("Tb", C.c_double), ("rimp", C.c_double), ("rbd", C.c_double), ("ni", C.c_double),
                ("meh", C.c_int), ("lp", C.c_int), ("beamf", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("beam_lx", C.c_double), ("beam_ly", C.c_double), ("beam_lz", C.c_double)]


class PicProfile(C.Structure):
    _fields_ = [("ppc_mean", C.c_double), ("cos_amp", C.c_double), ("bump_peak", C.c_double),
                ("bump_sigma", C.c_double), ("bump_centre", C.c_double * 3), ("count_seed", C.c_uint64)]


D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)
I32 = C.POINTER(C.c_int)
I64 = C.POINTER(C.c_int64)
H = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "pic_config_init": (None, [C.POINTER(PicConfig)]),
    "pic_create": (C.c_int, [C.POINTER(PicConfig), C.POINTER(C.c_void_p)]),
    "pic_destroy": (C.c_int, [H]),
    "pic_load_particles": (C.c_int, [H, C.c_int, C.c_int64] + [D] * 6 + [I64]),
    "pic_load_particles_device": (C.c_int, [H, C.c_int, C.c_int64] + [C.c_void_p] * 6 + [I64]),
    "pic_load_particles_cells": (C.c_int, [H, C.c_int, C.c_int64, C.c_void_p] + [C.c_void_p] * 6 + [I64]),
    "pic_get_particles_cells": (C.c_int, [H, C.c_int, C.c_int64, C.c_void_p] + [C.c_void_p] * 6 + [I64]),
    "pic_init_species_device": (C.c_int, [H, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.c_uint64]),
    "pic_init_species_host": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64] + [D] * 6),
    "pic_set_field": (C.c_int, [H, C.c_int, D]),
    "pic_get_field": (C.c_int, [H, C.c_int, D]),
    "pic_step": (C.c_int, [H, C.c_int]),
    "pic_run": (C.c_int, [H, C.c_int, D]),
    "pic_b_half": (C.c_int, [H]),
    "pic_stage_fields": (C.c_int, [H]),
    "pic_push_deposit": (C.c_int, [H]),
    "pic_migrate": (C.c_int, [H]),
    "pic_j_fold": (C.c_int, [H]),
    "pic_b_complete": (C.c_int, [H]),
    "pic_e_update": (C.c_int, [H]),
    "pic_e_ghosts": (C.c_int, [H]),
    "pic_get_cell_counts": (C.c_int, [H, I32]),
    "pic_get_cell_particles": (C.c_int, [H, C.c_int, C.c_int, C.c_int64] + [D] * 6 + [I64, I64, I64]),
    "pic_num_particles": (C.c_int64, [H, C.c_int]),
    "pic_get_particles": (C.c_int, [H, C.c_int, C.c_int64] + [D] * 6 + [I32, I64]),
    "pic_energy": (C.c_int, [H, D]),
    "pic_energy_reference": (C.c_int, [H, D]),
    "pic_charge_density": (C.c_int, [H, D]),
    "pic_gauss_residual": (C.c_int, [H, D]),
    "pic_gauss_check": (C.c_int, [H, C.c_int, D]),
    "pic_momentum": (C.c_int, [H, D]),
    "pic_mumu_name": (C.c_int, [C.c_int, C.c_int, C.c_char_p, C.c_int]),
    "pic_mumu_write": (C.c_int, [C.c_char_p, C.POINTER(PicMumu)]),
    "pic_mumu_read_counts": (C.c_int, [C.c_char_p, C.POINTER(PicMumu)]),
    "pic_mumu_read": (C.c_int, [C.c_char_p, C.POINTER(PicMumu)]),
    "pic_dump_write": (C.c_int, [H, C.c_char_p]),
    "pic_dump_read": (C.c_int, [H, C.c_char_p]),
    "pic_rnd_init": (None, [C.POINTER(PicRnd)]),
    "pic_rnd_uniform": (C.c_double, [C.POINTER(PicRnd)]),
    "pic_rnd_gaussian": (C.c_double, [C.POINTER(PicRnd), C.c_double, C.c_double]),
    "pic_rnd_table": (C.c_int, [D]),
    "pic_quiet_defaults": (C.c_int, [C.POINTER(PicQuiet)]),
    "pic_quiet_start": (C.c_int, [C.POINTER(PicQuiet)] + [C.POINTER(C.c_void_p)] * 3 + [I64, D, D]),
    "pic_profile_counts": (C.c_int, [C.c_int] * 3 + [C.POINTER(PicProfile), I32, I64]),
    "pic_init_species_profile": (C.c_int, [H, C.c_int, C.POINTER(PicProfile)] + [C.c_double] * 4 + [C.c_uint64]),
    "pic_sync": (C.c_int, [H]),
    "pic_last_status": (C.c_int, [H]),
    "pic_last_error_string": (C.c_char_p, [H]),
    "pic_error_string": (C.c_char_p, [C.c_int]),
    "pic_step_counters": (C.c_int, [H, I64]),
    "pic_step_timings": (C.c_int, [H, F]),
    "pic_layout_info": (C.c_int, [H, I64]),
    "pic_stream": (C.c_void_p, [H]),
    "pic_forward": (C.c_int, [H, C.c_int, C.c_int]),
    "pic_forward2": (C.c_int, [H, C.c_int, C.c_int, C.c_int]),
    "pic_branch_record": (C.c_int, [H, C.c_int]),
    "pic_forward_replay": (C.c_int, [H, C.c_int, H]),
    "pic_perturb_momenta": (C.c_int, [H, C.c_int, C.c_int64, D, C.c_double]),
    "pic_forward_history": (C.c_int, [H, D]),
    "pic_loss_value": (C.c_int, [H, C.POINTER(PicLoss), D]),
    "pic_backward": (C.c_int, [H, C.POINTER(PicLoss), C.POINTER(PicGrads)]),
    "pic_adjoint_timings": (C.c_int, [H, F]),
    "pic_adjoint_free": (C.c_int, [H]),
    "pic_field_energy_noalloc": (C.c_int, [C.c_int] * 3 + [C.c_void_p] * 8),
    # archAPI replacement (pic0buf_arch.h)
    "MemoryCopy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]),
    "MemoryAllocate": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    "GetDeviceMemory": (C.c_int, [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "MemorySet": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t]),
    "ThreadSynchronize": (C.c_int, []),
    "DeviceSynchronize": (C.c_int, []),
    "getLastError": (C.c_int, []),
    "getErrorString": (C.c_char_p, [C.c_int]),
    "SetDevice": (C.c_int, [C.c_int]),
}

_lib = None


def load() -> C.CDLL:
    """Load ``libpic0buf.so`` (building nothing).  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run python 0buf_b200/build.py)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class PicError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        name = PIC_ERR.get(status, f"cuda error {status}" if status > 0 else str(status))
        super().__init__(f"{where}: {name} ({detail})" if detail else f"{where}: {name}")


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(I32)
