"""The bench's multi-rank plumbing on CPU (gloo, world size 2): the
max/sum-over-ranks reductions the timing uses, and the reference arm under
torchrun, where rank 0 alone runs and prints one JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


RANK_SCRIPT = r"""
import importlib.util, json, os, sys
spec = importlib.util.spec_from_file_location("bench", os.path.join(sys.argv[1], "bench.py"))
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)
d = bench.Dist()
d.init("gloo")
r = d.rank
out = {"rank": r, "world": d.world, "max": d.max(10.0 + r), "sum": d.sum(1.5 * (r + 1))}
d.barrier()
d.close()
print(json.dumps(out), flush=True)
"""


def test_dist_reductions_gloo_world2(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=240)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max"] == 11.0
        assert o["sum"] == 4.5


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref0buf.so"))
                    and not os.path.exists(os.path.join(ROOT, "oracle", "lib", "libpicoracle.so")),
                    reason="no CPU implementation built")
def test_reference_arm_under_torchrun_world2():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--reference-inner", "1"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0
    assert out["e2e"]["h2d_bytes_per_step"] == 0


def test_bench_particle_matching():
    """bench.match_particles pairs the same generated particles held by two
    handles, one with FP32-rounded positions and in another order, including
    two particles of one cell whose x coincide after FP32 rounding (sorting
    alone swaps them)."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(1)
    n = 20000
    cell = rng.integers(0, 500, n)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    x[0], x[1], y[0], y[1], cell[1] = 0.5, 0.5 + 1e-9, 0.9, 0.1, cell[0]
    a = dict(cell=cell, x=x, y=y, z=z)
    perm = rng.permutation(n)
    b = {k: v[perm].copy() for k, v in a.items()}
    b["x"] = b["x"].astype(np.float32).astype(np.float64)
    ia, ib, repaired = bench.match_particles(a, b)
    assert np.array_equal(perm[ib], ia)
    assert repaired == 2
