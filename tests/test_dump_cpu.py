"""The reference's Fortran-record dump ("mumu" file) on the host: the
library's writer and reader (pic_mumu_write / pic_mumu_read) against the
oracle's numpy restatement of the format and against the reference's own
reader, LoadParticleData (load_data.cu:308-341), from the replay library."""
import os

import numpy as np
import pytest

from conftest import ROOT

CELLS = (6, 4, 5)
NODES = int(np.prod([c + 2 for c in CELLS]))
NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz", "Jx", "Jy", "Jz", "Qx", "Qy", "Qz")


def sample(seed=1, counts=(7, 11, 3)):
    rng = np.random.default_rng(seed)
    fields = {n: rng.normal(0, 1e-3, NODES) for n in NAMES}
    sorts = []
    for s, n in enumerate(counts):
        sp = {k: rng.uniform(0, 0.6, n) for k in ("x", "y", "z")}
        sp.update({k: rng.normal(0, 0.05, n) for k in ("px", "py", "pz")})
        sp.update(q_m=(1 / 1836, -1.0, -1.0)[s], m=(0.3, -0.25, -0.0025)[s])
        sorts.append(sp)
    return fields, sorts


def test_name(pkg):
    assert pkg.mumu_name(0, 42) == "mumu00000000042.dat"   # LoadParticleData's mumu000%08d.dat
    assert pkg.mumu_name(600, 7) == "mumu60000000007.dat"


def test_round_trip_and_numpy_restatement(pkg, oracle_mod, tmp_path):
    fields, sorts = sample()
    p = str(tmp_path / "a.dat")
    pkg.mumu_write(p, CELLS, fields, sorts)
    f2, s2 = pkg.mumu_read(p, CELLS)
    for n in NAMES:
        assert np.array_equal(f2[n], fields[n])
    assert len(s2) == 3
    for a, b in zip(sorts, s2):
        assert a["q_m"] == b["q_m"] and a["m"] == b["m"]
        for k in ("x", "y", "z", "px", "py", "pz"):
            assert np.array_equal(a[k], b[k])
    # the numpy restatement reads the library's file ...
    fn, sn = oracle_mod.read_mumu_np(p, CELLS)
    assert all(np.array_equal(fn[i], fields[n]) for i, n in enumerate(NAMES))
    assert np.array_equal(sn[1][2], sorts[1]["x"])
    # ... and the library reads the restatement's file
    q = str(tmp_path / "b.dat")
    oracle_mod.write_mumu_np(q, CELLS, [fields[n] for n in NAMES],
                             [(sp["q_m"], sp["m"], *[sp[k] for k in ("x", "y", "z", "px", "py", "pz")]) for sp in sorts])
    assert open(p, "rb").read() == open(q, "rb").read()


def test_missing_fields_are_zero_and_empty_sorts(pkg, tmp_path):
    p = str(tmp_path / "c.dat")
    fields, sorts = sample(counts=(0, 5, 0))
    pkg.mumu_write(p, CELLS, {"Ex": fields["Ex"]}, sorts)
    f2, s2 = pkg.mumu_read(p, CELLS)
    assert np.array_equal(f2["Ex"], fields["Ex"]) and not f2["Qz"].any()
    assert [s["x"].size for s in s2] == [0, 5, 0]


def test_malformed_files_are_rejected(pkg, tmp_path):
    fields, sorts = sample()
    p = str(tmp_path / "d.dat")
    pkg.mumu_write(p, CELLS, fields, sorts)
    raw = open(p, "rb").read()
    bad = str(tmp_path / "bad.dat")
    open(bad, "wb").write(raw[:-3])                   # truncated
    with pytest.raises(pkg.PicError):
        pkg.mumu_read(bad, CELLS)
    corrupt = bytearray(raw)
    corrupt[4 + NODES * 8] ^= 1                      # first record's closing marker
    open(bad, "wb").write(bytes(corrupt))
    with pytest.raises(pkg.PicError):
        pkg.mumu_read(bad, CELLS)
    with pytest.raises(pkg.PicError):                # another grid
        pkg.mumu_read(p, (6, 4, 4))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref0buf.so")),
                    reason="needs the reference replay library (oracle/build_ref.sh)")
def test_reference_reader_reads_the_library_dump(pkg, oracle_mod, tmp_path):
    """The library writes mumu00000000007.dat; the reference's own
    LoadParticleData reads its three sorts back with every value intact."""
    fields, sorts = sample(seed=4, counts=(9, 13, 4))
    pkg.mumu_write(str(tmp_path / pkg.mumu_name(0, 7)), CELLS, fields, sorts)
    got = oracle_mod.ref_read_mumu(str(tmp_path), 7, CELLS)
    assert [g.shape[0] for g in got] == [9, 13, 4]
    for sp, g in zip(sorts, got):
        for a, k in enumerate(("x", "y", "z", "px", "py", "pz")):
            assert np.array_equal(g[:, a], sp[k]), k
        assert np.all(g[:, 6] == sp["m"]) and np.all(g[:, 7] == sp["q_m"])
