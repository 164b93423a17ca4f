"""The oracle (oracle/hmvm_oracle.c) pinned to the reference's own outputs.

* golden vectors under tests/golden/ were produced by the reference's
  hmvm_seq_2 (see make_golden.py): the oracle must reproduce them bit for bit;
* where the reference build oracle/_ref exists, the oracle is compared with it
  directly (seq_2 both loop orders, float mode, omp_2);
* on the reference's shipped hmatrix_sample.bin when it is present.
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix
from helpers import (GOLDEN, SAMPLE_BIN, RefMatrix, oracle_hmvm, oracle_lib, oracle_omp, ref_available, ref_lib,
                     relerr)

META = json.load(open(os.path.join(GOLDEN, "golden.json")))
Y = np.load(os.path.join(GOLDEN, "golden_y.npz"))


def _orc_load(path, fmt=1):
    """Load with the oracle's own restated loader (64-bit offsets)."""
    lib = oracle_lib()
    rc = C.c_int()
    h = lib.orc_open(path.encode(), fmt, C.byref(rc))
    assert h, rc.value
    info = np.zeros(4, np.int64)
    lib.orc_info(h, info.ctypes.data_as(C.c_void_p))
    nd, nlf, ktmax, ln = (int(v) for v in info)
    arrs = [np.zeros(nlf, np.int32) for _ in range(6)] + [np.zeros(nlf, np.int64) for _ in range(2)] + [np.zeros(ln)]
    lib.orc_export(h, *[a.ctypes.data_as(C.c_void_p) for a in arrs])
    lib.orc_close(h)
    lt, kt, ndl, ndt, sl, st, a1, a2, rm = arrs
    return HMatrix.from_arrays(nd, ktmax, lt, kt, ndl, ndt, sl, st, a1, a2, rm)


@pytest.mark.parametrize("name", sorted(META["matrices"]))
def test_oracle_reproduces_reference_golden(name):
    m = META["matrices"][name]
    path = os.path.join(GOLDEN, m["file"])
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == m["sha256"]
    hm = _orc_load(path)
    assert (hm.nd, hm.nlf, hm.ktmax, hm.len) == (m["nd"], m["nlf"], m["ktmax"], m["len"])
    for xn in ("sin", "uniform"):
        x = Y[f"{name}/x_{xn}"]
        assert np.array_equal(oracle_hmvm(hm, x, 0), Y[f"{name}/y_seq2_d_{xn}"])
        assert np.array_equal(oracle_hmvm(hm, x, 1), Y[f"{name}/y_seq2i_d_{xn}"])
        yf = oracle_hmvm(hm.to_float(), x.astype(np.float32), 0)
        assert np.array_equal(yf, Y[f"{name}/y_seq2_f_{xn}"])


def test_known_answer_is_exact():
    from make_golden import kat_matrix

    hm = kat_matrix()
    x = Y["kat6/x_uniform"]
    A = hm.dense()
    assert np.array_equal(oracle_hmvm(hm, np.arange(1.0, 7.0)), A @ np.arange(1.0, 7.0))
    assert relerr(oracle_hmvm(hm, x), A @ x) < 1e-15


def test_omp_restatement_matches_sequential():
    hm = _orc_load(os.path.join(GOLDEN, META["matrices"]["cube300"]["file"]))
    x = Y["cube300/x_sin"]
    # hmvm_omp_2 merges per-thread partial vectors: equal up to rounding order
    for nt in (1, 3, 8):
        assert relerr(oracle_omp(hm, x, nt), Y["cube300/y_seq2_d_sin"]) < 1e-14


@pytest.mark.skipif(not ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("case", [(700, "sphere", 2.0, 1e-4, 32, 1), (900, "cube", 1.0, 1e-6, 20, 2),
                                  (500, "plate", 2.0, 1e-3, 12, 3)])
def test_oracle_equals_reference_build(case):
    n, geo, eta, eps, leaf, seed = case
    hm = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=seed)
    ref = RefMatrix(hm)
    for seed_x in (0, 1):
        x = np.random.default_rng(seed_x).uniform(-1, 1, n)
        for a2i in (0, 1):
            assert np.array_equal(oracle_hmvm(hm, x, a2i), ref.seq2(x, a2i))
        xf = x.astype(np.float32)
        assert np.array_equal(oracle_hmvm(hm.to_float(), xf), ref.seq2_f(xf))
        assert relerr(ref.omp2(x), ref.seq2(x)) < 1e-14
    ref.close()


@pytest.mark.skipif(not os.path.exists(SAMPLE_BIN), reason="reference sample matrix absent")
def test_reference_sample_matrix():
    s = META["sample"]
    assert s is not None
    assert hashlib.sha256(open(SAMPLE_BIN, "rb").read()).hexdigest() == s["sha256"]
    hm = _orc_load(SAMPLE_BIN)
    assert (hm.nd, hm.nlf, hm.ktmax, hm.len) == (s["nd"], s["nlf"], s["ktmax"], s["len"]) == (600, 1426, 31, 248662)
    x = np.sin(np.arange(1, hm.nd + 1, dtype=np.float64))
    assert np.array_equal(oracle_hmvm(hm, x), Y["sample/y_seq2_d_sin"])
    assert np.array_equal(Y["sample/y_seq1_d_sin"], Y["sample/y_seq2_d_sin"])  # AoS == SoA in the reference
    xf = np.sin(np.arange(1, hm.nd + 1, dtype=np.float32))
    assert np.array_equal(oracle_hmvm(hm.to_float(), xf), Y["sample/y_seq2_f_sin"])
    # the shipped sample's structure: 210 low-rank and 1216 dense leaves, ranks 10..31
    lr = hm.ltmtx == 1
    assert int(lr.sum()) == 210 and int((~lr).sum()) == 1216
    assert hm.kt[lr].min() == 10 and hm.kt[lr].max() == 31
    assert np.all(np.diff(hm.nstrtl) >= 0)
    if ref_available():
        lib = ref_lib()
        h = lib.ref_load1(SAMPLE_BIN.encode())
        y = np.empty(hm.nd)
        lib.ref_seq2_d(h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0)
        lib.ref_free(h)
        assert np.array_equal(y, Y["sample/y_seq2_d_sin"])


def test_oracle_loaders_agree_bin1_bin2(tmp_path):
    hm = HMatrix.generate(600, "cube", eps=1e-4, leaf_size=16, seed=5)
    p1, p2 = str(tmp_path / "h1.bin"), str(tmp_path / "h2.bin")
    hm.write_bin1(p1)
    hm.write_bin2(p2)
    a, b = _orc_load(p1, 1), _orc_load(p2, 2)
    for f in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2", "rowmat"):
        assert np.array_equal(getattr(a, f), getattr(hm, f)), f
        assert np.array_equal(getattr(b, f), getattr(hm, f)), f


def test_oracle_loader_rejects_corrupt_files(tmp_path):
    lib = oracle_lib()
    p = str(tmp_path / "h.bin")
    HMatrix.generate(300, "sphere", leaf_size=16, seed=3).write_bin1(p)
    raw = open(p, "rb").read()
    rc = C.c_int()
    # truncated in a leaf record, truncated early, and a broken closing marker of the header record
    for bad in (raw[:-7], raw[:100], raw[:16] + b"\xff\xff\xff\x7f" + raw[20:]):
        q = str(tmp_path / "bad.bin")
        open(q, "wb").write(bad)
        assert not lib.orc_open(q.encode(), 1, C.byref(rc))
        assert rc.value < 0
    assert not lib.orc_open(str(tmp_path / "missing.bin").encode(), 1, C.byref(rc))
    assert rc.value == -1
