"""C ABI checks that need no GPU: the library loads, exports every symbol
the public headers declare, validates arguments, and the host generator is
deterministic and places every particle strictly inside its cell."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available


def declared_functions():
    names = set()
    for hdr in ("pic0buf.h", "pic0buf_arch.h"):
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                             src, flags=re.M):
            if m.group(1) not in ("if", "while", "return", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load_library()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header(pkg):
    from importlib import import_module
    capi = import_module("0buf_b200._capi")
    assert set(declared_functions()) <= set(capi.SIGNATURES)


def test_config_validation_without_gpu(pkg):
    lib = pkg.load_library()
    capi = pkg._capi
    cfg = capi.PicConfig()
    lib.pic_config_init(C.byref(cfg))
    assert cfg.precision == capi.PIC_FP64_PLAIN and cfg.capacity_pad == -1
    h = C.c_void_p()
    cfg.nx, cfg.ny, cfg.nz = 2, 4, 4  # fewer than 3 cells on an axis
    cfg.lx = cfg.ly = cfg.lz = 0.4
    cfg.tau = 0.02
    cfg.nspecies = 1
    cfg.species[0].q_m = -1.0
    cfg.species[0].m = -0.1
    assert lib.pic_create(C.byref(cfg), C.byref(h)) == -1
    cfg.nx = 4
    cfg.tau = -1.0
    assert lib.pic_create(C.byref(cfg), C.byref(h)) == -1
    cfg.tau = 0.02
    cfg.species[0].q_m = 0.0
    assert lib.pic_create(C.byref(cfg), C.byref(h)) == -1


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU path")
def test_no_device_fails_loudly(pkg):
    with pytest.raises(pkg.PicError) as e:
        pkg.PicSimulation((4, 4, 4), (0.4, 0.4, 0.4), 0.02, [(-1.0, -0.1, 1)])
    assert e.value.status == -9


def test_error_strings(pkg):
    lib = pkg.load_library()
    assert lib.pic_error_string(0) == b"success"
    assert b"half a cell" in lib.pic_error_string(-3)
    assert lib.pic_error_string(-513131313) == b"too many particles"


def test_arch_layer_direction_check(pkg):
    lib = pkg.load_library()
    a = (C.c_char * 8)()
    b = (C.c_char * 8)()
    # an unknown direction code is rejected before any CUDA call (archAPI.cu:44-53 leaves it uninitialised)
    assert lib.MemoryCopy(C.cast(a, C.c_void_p), C.cast(b, C.c_void_p), 8, 12345) == 21
    assert lib.getErrorString(0) == b"no error"


def test_host_generator_deterministic_and_inside(pkg):
    cells, lengths = (6, 5, 4), (0.6, 0.5, 0.4)
    a = pkg.host_species(cells, lengths, 1, 7, (0.0, 0.0, 0.0), 0.02, 5)
    b = pkg.host_species(cells, lengths, 1, 7, (0.0, 0.0, 0.0), 0.02, 5)
    c = pkg.host_species(cells, lengths, 1, 7, (0.0, 0.0, 0.0), 0.02, 6)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    assert not np.array_equal(a[0], c[0])
    n = int(np.prod(cells)) * 7
    x, y, z = a[0], a[1], a[2]
    h = [L / N for L, N in zip(lengths, cells)]
    idx = np.arange(n) // 7
    ci, cl, ck = idx // (cells[1] * cells[2]), (idx // cells[2]) % cells[1], idx % cells[2]
    for pos, cc, hh in ((x, ci, h[0]), (y, cl, h[1]), (z, ck, h[2])):
        # getPointCell (cell.h:593-598) and isPointInCell (cell.h:717) agree with the slot's cell
        assert np.array_equal((pos / hh).astype(np.int64), cc)
        x0 = cc * hh
        assert np.all((x0 <= pos) & (pos < x0 + hh))


def test_host_generator_moments(pkg):
    cells, lengths = (8, 8, 8), (0.8, 0.8, 0.8)
    x, y, z, px, py, pz = pkg.host_species(cells, lengths, 2, 64, (0.2, 0.0, 0.0), 0.002, 1)
    assert abs(px.mean() - 0.2) < 1e-4 and abs(py.mean()) < 1e-4
    assert abs(px.std() - 0.002) < 5e-5 and abs(pz.std() - 0.002) < 5e-5
    # uniform in-cell offsets
    ox = (x / 0.1) % 1.0
    assert abs(ox.mean() - 0.5) < 0.01
    cold = pkg.host_species(cells, lengths, 0, 4, (0.0, 0.0, 0.0), 0.0, 1)
    assert not cold[3].any() and not cold[4].any() and not cold[5].any()


def test_configs(pkg):
    c = pkg.configs
    assert c.CONFIGS["c2"]["cells"] == (512, 128, 128)
    t = c.species_table(32)
    assert t[0][1] == pytest.approx(1.01 / 32) and t[1][1] == pytest.approx(-1.0 / 32)
    assert t[2][1] == pytest.approx(-0.01 / 32)
    n = np.prod(c.CONFIGS["c2"]["cells"]) * 3 * c.CONFIGS["c2"]["ppc"]
    assert n == 805306368


def test_profile_counts(pkg):
    """The stress configuration's density profile: mean ppc, cos modulation in
    x, the bump at the box centre, identical counts for the same count seed."""
    cells = (32, 16, 16)
    prof = dict(pkg.configs.C4_PROFILE, ppc_mean=20)
    n = pkg.profile_counts(cells, prof)
    assert n.shape == cells
    assert abs(n.mean() - 20) < 0.05
    assert n[15:17, 7:9, 7:9].max() >= n.max() - 1 and n.max() > 2 * 20
    assert np.array_equal(n, pkg.profile_counts(cells, prof))
    other = pkg.profile_counts(cells, dict(prof, count_seed=prof["count_seed"] + 1))
    assert not np.array_equal(n, other) and abs(other.mean() - 20) < 0.05
    flat = pkg.profile_counts(cells, dict(ppc_mean=20, cos_amp=0.5, bump_peak=1.0))
    # 1 + 0.5 cos(2 pi (i + 1/2) / Nx): densest at i = 0, thinnest at i = Nx/2
    assert flat[0].mean() > 1.4 * 20 and flat[16].mean() < 0.6 * 20
    with pytest.raises(pkg.PicError):
        pkg.profile_counts(cells, dict(ppc_mean=20, bump_peak=2.0, bump_sigma=0.0))
