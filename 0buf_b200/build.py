"""Build the CUDA library of the B200 PIC step into ``0buf_b200/lib/libpic0buf.so``.

Every translation unit is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``).  The FP64 parity code (plain
form, binning, C ABI) is compiled with ``-fmad=false`` so its arithmetic is the
reference's separate IEEE multiplies and adds; the FP32 mixed form keeps FMA
and flushes FP32 subnormals (``-ftz=true``: no subnormal handling around the
reciprocal square roots and divisions of its push).
The CUDA runtime is linked statically so the ``.so`` is self-contained.

Usage: ``python 0buf_b200/build.py [--force] [-j N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libpic0buf.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC] + ARCH

# translation unit -> extra flags
UNITS = {
    "pic_plain.cu": ["-fmad=false"],
    "pic_common.cu": ["-fmad=false"],
    "pic_capi.cu": ["-fmad=false"],
    "pic_arch.cu": [],
    "pic_mixed.cu": ["-ftz=true"],
    "pic_noalloc.cu": [],
    "pic_diag.cu": ["-fmad=false"],
    "pic_dump.cu": [],
    "pic_quiet.cu": ["-Xcompiler", "-ffp-contract=off"],
    "pic_adjoint.cu": ["-fmad=false"],
    "pic_adjoint_mixed.cu": [],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def compile_unit(name: str, flags: list[str], force: bool, verbose: bool) -> str:
    src = os.path.join(CSRC, name)
    obj = os.path.join(OBJ, name.replace(".cu", ".o"))
    if force or _stale(obj, [src, __file__] + _headers()):
        cmd = [nvcc()] + COMMON + flags + ["-c", src, "-o", obj + ".tmp"]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    jobs = jobs or min(len(UNITS), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(compile_unit, n, f, force, verbose) for n, f in UNITS.items()]
        objs = [f.result() for f in futs]
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("-v", action="store_true", help="print ptxas register/spill info")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    main()
