"""The library's loaders (hmvm_b200_load_hmatrix / _load_hmatrix2 /
_convert_d2f, replacing src_hmvm/src_cpp/loadmatrix.cpp): same results as the
reference's own loaders, and status codes instead of crashes on bad files."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import GOLDEN, SAMPLE_BIN, ref_available, ref_lib

LIB = None


def lib():
    global LIB
    if LIB is None:
        LIB = _lib.hmvm_lib()
    return LIB


def _np(ptr, n, dt):
    return np.ctypeslib.as_array(ptr, (n,)).view(dt).copy() if n else np.zeros(0, dt)


def load1(path, with_aos=True):
    m1, m2 = _lib.Matrix_d(), _lib.Matrix2_d()
    rc = lib().hmvm_b200_load_hmatrix(path.encode(), C.byref(m1) if with_aos else None, C.byref(m2))
    return rc, m1, m2


def soa(m2):
    n = m2.nlf
    return {f: _np(getattr(m2, f), n, np.int32) for f in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2")} | {
        "rowmat": _np(m2.rowmat, m2.len, np.float64), "rowmat_t": _np(m2.rowmat_t, m2.len, np.float64)}


def ref_soa(path, fmt):
    r = ref_lib()
    h = r.ref_load1(path.encode()) if fmt == 1 else r.ref_load2(path.encode())
    info = np.zeros(4, np.int32)
    r.ref_info(h, info.ctypes.data)
    nd, nlf, ktmax, ln = (int(v) for v in info)
    arrs = [np.zeros(nlf, np.int32) for _ in range(8)] + [np.zeros(ln)]
    r.ref_export2(h, *[a.ctypes.data for a in arrs])
    r.ref_free(h)
    names = ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2", "rowmat")
    return (nd, nlf, ktmax, ln), dict(zip(names, arrs))


def files():
    out = [os.path.join(GOLDEN, f) for f in sorted(os.listdir(GOLDEN)) if f.endswith("_hmatrix_1.bin")]
    if os.path.exists(SAMPLE_BIN):
        out.append(SAMPLE_BIN)
    return out


@pytest.mark.parametrize("path", files(), ids=os.path.basename)
def test_load1_matches_reference(path):
    rc, m1, m2 = load1(path)
    assert rc == 0, lib().hmvm_b200_last_error()
    try:
        got = soa(m2)
        # rowmat_t: U transposed to [ndl][kt], everything else copied (loadmatrix.cpp:227-234)
        for i in range(m2.nlf):
            if got["ltmtx"][i] == 1:
                k, l, a2 = got["kt"][i], got["ndl"][i], got["a2"][i]
                U = got["rowmat"][a2:a2 + k * l].reshape(k, l)
                assert np.array_equal(got["rowmat_t"][a2:a2 + k * l].reshape(l, k), U.T)
                sub = m1.submat[i]
                assert np.array_equal(np.ctypeslib.as_array(sub.a2t, (k * l,)), U.T.ravel())
        if ref_available():
            (nd, nlf, ktmax, ln), ref = ref_soa(path, 1)
            assert (m2.nd, m2.nlf, m2.ktmax, m2.len) == (nd, nlf, ktmax, ln)
            for f, v in ref.items():
                assert np.array_equal(got[f], v), f
    finally:
        lib().hmvm_b200_free_matrix_d(C.byref(m1))
        lib().hmvm_b200_free_matrix2_d(C.byref(m2))


def test_writer_roundtrip_and_bin2(tmp_path):
    hm = HMatrix.generate(900, "plate", eta=1.0, eps=1e-4, leaf_size=20, seed=8)
    p1, p2 = str(tmp_path / "hmatrix_1.bin"), str(tmp_path / "hmatrix_2.bin")
    hm.write_bin1(p1)
    hm.write_bin2(p2)
    for p, fmt in ((p1, 1), (p2, 2)):
        back = HMatrix.load(p)
        for f in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2", "rowmat"):
            assert np.array_equal(getattr(back, f), getattr(hm, f)), (fmt, f)
        if ref_available():
            _, ref = ref_soa(p, fmt)
            assert np.array_equal(ref["rowmat"], hm.rowmat)


def test_convert_d2f_matches_reference_cast():
    path = os.path.join(GOLDEN, "cube300_hmatrix_1.bin")
    rc, m1, m2 = load1(path)
    assert rc == 0
    f1, f2 = _lib.Matrix_f(), _lib.Matrix2_f()
    assert lib().hmvm_b200_convert_d2f(C.byref(f1), C.byref(f2), C.byref(m1), C.byref(m2)) == 0
    rm = _np(m2.rowmat, m2.len, np.float64)
    assert np.array_equal(_np(f2.rowmat, f2.len, np.float32), rm.astype(np.float32))
    assert np.array_equal(_np(f2.rowmat_t, f2.len, np.float32), _np(m2.rowmat_t, m2.len, np.float64).astype(np.float32))
    assert f2.nd == m2.nd and f2.nlf == m2.nlf and f2.ktmax == m2.ktmax
    s = f1.submat[1]
    assert s.ltmtx == m1.submat[1].ltmtx
    lib().hmvm_b200_free_matrix_f(C.byref(f1))
    lib().hmvm_b200_free_matrix2_f(C.byref(f2))
    lib().hmvm_b200_free_matrix_d(C.byref(m1))
    lib().hmvm_b200_free_matrix2_d(C.byref(m2))


def _records(raw):
    """Split a Fortran unformatted file into (offset, length) of payloads."""
    out, pos = [], 0
    while pos < len(raw):
        (n,) = struct.unpack_from("<i", raw, pos)
        out.append((pos + 4, n))
        pos += 8 + n
    return out


@pytest.mark.parametrize("fault", ["missing", "truncated", "bad_marker", "ltmtx", "row_range", "kt_gt_ktmax",
                                   "len_mismatch"])
def test_faults_return_status(tmp_path, fault):
    """Host-side fault injection: every bad input gives a status code (the
    reference would read garbage or exit)."""
    src = os.path.join(GOLDEN, "sphere256_hmatrix_1.bin")
    raw = bytearray(open(src, "rb").read())
    recs = _records(bytes(raw))
    p = str(tmp_path / "bad.bin")
    fmt = 1
    if fault == "missing":
        p = str(tmp_path / "does_not_exist.bin")
        want = _lib.HMVM_EIO
    elif fault == "truncated":
        raw = raw[: len(raw) // 2]
        want = _lib.HMVM_EFORMAT
    elif fault == "bad_marker":
        off, n = recs[3]
        struct.pack_into("<i", raw, off + n, n + 8)  # closing marker disagrees
        want = _lib.HMVM_EFORMAT
    elif fault in ("ltmtx", "row_range", "kt_gt_ktmax"):
        off, n = recs[1]  # first leaf header: ltmtx, ndl, ndt, nstrtl, nstrtt, kt
        vals = list(struct.unpack_from("<6i", raw, off))
        if fault == "ltmtx":
            vals[0] = 3
        elif fault == "row_range":
            vals[3] = 256  # nstrtl + ndl - 1 > nd
        else:
            vals[5] = 10 ** 6
            vals[0] = 1
        struct.pack_into("<6i", raw, off, *vals)
        want = _lib.HMVM_EFORMAT
    else:  # len_mismatch in hmatrix_2.bin
        hm = HMatrix.load(src)
        p2 = str(tmp_path / "h2.bin")
        hm.write_bin2(p2)
        raw = bytearray(open(p2, "rb").read())
        struct.pack_into("<i", raw, 4 + 12, hm.len + 5)
        fmt = 2
        want = _lib.HMVM_EFORMAT
    if fault != "missing":
        open(p, "wb").write(bytes(raw))
    m2 = _lib.Matrix2_d()
    if fmt == 1:
        m1 = _lib.Matrix_d()
        rc = lib().hmvm_b200_load_hmatrix(p.encode(), C.byref(m1), C.byref(m2))
    else:
        rc = lib().hmvm_b200_load_hmatrix2(p.encode(), C.byref(m2))
    assert rc == want, (rc, lib().hmvm_b200_last_error())
    assert lib().hmvm_b200_last_error()
    assert not m2.rowmat  # nothing handed back on failure
