"""A C++ client of the C ABI compiles and links against the library, and the
ABI structs it sees (sizes and field offsets from the C++ compiler) are the
ones the ctypes mirror (0buf_b200/_capi.py) declares."""
import ctypes as C
import subprocess

import pytest

from capi_client_build import build


def test_cpp_client_layout_matches_ctypes(pkg, tmp_path):
    cap = pkg._capi
    exe = build(str(tmp_path))
    out = subprocess.run([exe, "layout"], capture_output=True, text=True, check=True).stdout
    got = {ln.split()[0]: [int(v) for v in ln.split()[1:]] for ln in out.strip().splitlines()}

    def off(struct, *names):
        return [getattr(struct, n).offset for n in names]

    want = {
        "pic_species": [C.sizeof(cap.PicSpecies)] + off(cap.PicSpecies, "q_m", "m", "sort"),
        "pic_config": [C.sizeof(cap.PicConfig)] + off(cap.PicConfig, "nx", "ny", "nz", "lx", "ly", "lz", "tau",
                                                       "precision", "ghosts", "nspecies", "device", "species",
                                                       "capacity_slack", "outbox_fraction", "tile", "capacity_pad"),
        "pic_loss": [C.sizeof(cap.PicLoss)] + off(cap.PicLoss, "field", "window", "species", "drift", "vth"),
        "pic_grads": [C.sizeof(cap.PicGrads)] + off(cap.PicGrads, "loss", "d_drift", "d_vth", "n", "d_p0"),
        "pic_profile": [C.sizeof(cap.PicProfile)],
        "pic_mumu": [C.sizeof(cap.PicMumu)] + off(cap.PicMumu, "fields", "count", "q_m", "m", "p"),
        "pic_rnd": [C.sizeof(cap.PicRnd)] + off(cap.PicRnd, "store"),
        "pic_quiet": [C.sizeof(cap.PicQuiet)] + off(cap.PicQuiet, "meh", "lx"),
    }
    assert got == want


def test_cpp_client_usage(tmp_path):
    exe = build(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
