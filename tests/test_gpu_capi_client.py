"""The C++ client (tests/capi_client.cpp: the reference's Plasma step driver
over the C ABI, built with g++) runs the reference fixture's small case on the
GPU: per-cell counts identical to the reference's every step, fields within
1e-12 relative L2 and the reference's electric energy within 1e-12."""
import os
import subprocess

import numpy as np
import pytest

from capi_client_build import build
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIELDS = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz"]


def rel_l2(a, b):
    d = np.linalg.norm(a - b)
    return 0.0 if d == 0.0 else d / max(np.linalg.norm(b), 1e-300)


def test_cpp_client_runs_reference_case(tmp_path):
    d = np.load(os.path.join(GOLDEN, "ref_small.npz"))
    cells = [int(c) for c in d["cells"]]
    h, tau, steps = float(d["h"]), float(d["tau"]), int(d["steps"])
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(np.array(cells + [3, steps], dtype=np.int32).tobytes())
        f.write(np.array([c * h for c in cells] + [tau], dtype=np.float64).tobytes())
        for s in range(3):
            x = d[f"in_s{s}_x"]
            f.write(np.array([d[f"in_s{s}_q_m"], d[f"in_s{s}_m"]], dtype=np.float64).tobytes())
            f.write(np.array([x.size], dtype=np.int64).tobytes())
            for k in ("x", "y", "z", "px", "py", "pz"):
                f.write(np.ascontiguousarray(d[f"in_s{s}_{k}"], dtype=np.float64).tobytes())
        for fld in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            f.write(np.ascontiguousarray(d[f"in_{fld}"], dtype=np.float64).tobytes())
    exe = build(str(tmp_path))
    r = subprocess.run([exe, "run", str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nodes = int(np.prod([c + 2 for c in cells]))
    raw = open(out, "rb").read()
    per = nodes * 4 + 12 * nodes * 8 + 8
    assert len(raw) == steps * per
    for st in range(1, steps + 1):
        base = (st - 1) * per
        counts = np.frombuffer(raw, np.int32, nodes, base)
        assert np.array_equal(counts, d[f"step{st}_counts"]), st
        for i, fld in enumerate(FIELDS):
            a = np.frombuffer(raw, np.float64, nodes, base + nodes * 4 + i * nodes * 8)
            assert rel_l2(a, d[f"step{st}_{fld}"]) <= 1e-12, (st, fld)
        e = np.frombuffer(raw, np.float64, 1, base + nodes * 4 + 12 * nodes * 8)[0]
        assert e == pytest.approx(float(d[f"step{st}_energy"]), rel=1e-12)
