"""Builds tests/capi_client.cpp (a C++ client of include/pic0buf.h) with g++
against 0buf_b200/lib/libpic0buf.so; used by the CPU and GPU tests."""
import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "capi_client.cpp")
LIBDIR = os.path.join(ROOT, "0buf_b200", "lib")


def build(outdir: str) -> str:
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        raise RuntimeError("no C++ compiler")
    exe = os.path.join(outdir, "capi_client")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", exe, "-L", LIBDIR, "-lpic0buf", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{r.stdout}\n{r.stderr}")
    return exe
