"""B200-native (sm_100a) 3D electromagnetic PIC time step of snytav/0buf.

The package directory starts with a digit, so import it with
``importlib.import_module("0buf_b200")``.  The compute path is the CUDA library
``lib/libpic0buf.so`` (C ABI in ``include/pic0buf.h``); this package is the
host-side mirror of the reference's step driver over that ABI.
"""
from . import _capi, configs, compare
from ._capi import PicError, load as load_library, LIB_PATH
from .plasma import (PicSimulation, Plasma, Rnd, host_species, profile_counts, mumu_name, mumu_read, mumu_write,
                     quiet_params, quiet_start)

__all__ = ["PicSimulation", "Plasma", "PicError", "host_species", "profile_counts", "mumu_name", "mumu_read",
           "mumu_write", "Rnd", "quiet_params", "quiet_start", "load_library", "LIB_PATH", "configs", "compare"]
