"""pic_field_energy_noalloc (no allocation, static device scratch) against
pic_energy / pic_energy_reference of the same fields, through the C ABI.

Two calls in a row on different field states: the scratch keeps the first
call's partial sums, and the second result must not depend on them.  Collected
last on purpose, so it also runs after every other test in one process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12  # relative; only the order of the FP64 sums differs
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _noalloc_energy(lib, torch, sim, cells):
    dev = [torch.from_numpy(np.ascontiguousarray(sim.get_field(f))).cuda() for f in FIELDS]
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.pic_field_energy_noalloc(*cells, *[t.data_ptr() for t in dev], out.data_ptr(), None)
    assert rc == 0, lib.pic_error_string(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check(sim, got):
    want = sim.energy()
    np.testing.assert_allclose(got[0], want[0], rtol=REL, atol=0)
    np.testing.assert_allclose(got[1], want[1], rtol=REL, atol=0)
    np.testing.assert_allclose(got[2], sim.energy_reference(), rtol=REL, atol=0)


def test_field_energy_noalloc_matches(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = pkg._capi.load()
    cells = (16, 8, 8)
    table = [(1.0 / 1836.0, 1.01 / 4, 0), (-1.0, -1.0 / 4, 1), (-1.0, -0.01 / 4, 2)]
    with pkg.PicSimulation(cells, tuple(0.2 * c for c in cells), 0.05, table, precision="fp64") as sim:
        sim.init_species(0, 4, seed=1)
        sim.init_species(1, 4, vth=0.05, seed=2)
        sim.init_species(2, 4, drift=(0.2, 0.0, 0.0), vth=0.01, seed=3)
        sim.run(3)
        first = _noalloc_energy(lib, torch, sim, cells)
        assert first[0] > 0 and first[1] > 0
        _check(sim, first)
        sim.run(2)
        second = _noalloc_energy(lib, torch, sim, cells)
        assert not np.array_equal(first, second)
        _check(sim, second)

        # on a caller's own stream: enqueued there, ready once that stream is synchronised
        stream = torch.cuda.Stream()
        dev = [torch.from_numpy(np.ascontiguousarray(sim.get_field(f))).cuda() for f in FIELDS]
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.pic_field_energy_noalloc(*cells, *[t.data_ptr() for t in dev], out.data_ptr(),
                                          C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.pic_error_string(rc)
        stream.synchronize()
        _check(sim, out.cpu().numpy())

        # a grid beyond the static scratch is refused before any device work
        rc = lib.pic_field_energy_noalloc(2 ** 31 - 2, 4, 4, *([C.c_void_p(1)] * 7), None)
        assert pkg._capi.PIC_ERR.get(rc) == "PIC_ERR_ARG"
        rc = lib.pic_field_energy_noalloc(4096, 4096, 4096, *([C.c_void_p(1)] * 7), None)
        assert pkg._capi.PIC_ERR.get(rc) == "PIC_ERR_ARG"
