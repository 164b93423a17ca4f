"""The 64-bit variant of hmatrix_2.bin and the 64-bit loader
(hmvm_b200_load_leaves64, hgen_write_bin64): the dump layout of
HACApK_hdump_dump_leafmtx2 (src_hdump/m_HACApK_hdump.f90:114-180) with the
header's len as int64, which lifts the int len / a1 / a2 ceiling of
loadHmatrix2 (src_hmvm/src_cpp/hacapk.h:28,31; loadmatrix.cpp:152-250).

* CPU: every format round-trips through the 64-bit loader to the same arrays the
  reference-signature loaders give; the header's len is read as 64 bits; bad
  files give status codes.
* GPU: a file of more than 2^31 elements (a sparse file: a few non-zeros, holes
  elsewhere) loads, plans and multiplies with its offsets past 2^31 intact.
"""
import ctypes as C
import os
import struct

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan, _lib
from helpers import oracle_hmvm, relerr

FIELDS = ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2", "rowmat")


@pytest.fixture(scope="module")
def hm():
    return HMatrix.generate(1200, "cube", eta=2.0, eps=1e-4, leaf_size=24, seed=12)


def test_formats_roundtrip_wide(hm, tmp_path):
    paths = {1: str(tmp_path / "h1.bin"), 2: str(tmp_path / "h2.bin"), 3: str(tmp_path / "h64.bin")}
    hm.write_bin1(paths[1])
    hm.write_bin2(paths[2])
    hm.write_bin64(paths[3])
    # the 64-bit header record is 20 bytes: nd, nlf, ktmax (int32), len (int64)
    raw = open(paths[3], "rb").read(28)
    assert struct.unpack_from("<i3iqi", raw) == (20, hm.nd, hm.nlf, hm.ktmax, hm.len, 20)
    # apart from that header the files are byte-identical to bin2
    assert open(paths[3], "rb").read()[28:] == open(paths[2], "rb").read()[24:]
    x = np.random.default_rng(2).uniform(-1, 1, hm.nd)
    y0 = oracle_hmvm(hm, x)
    for fmt, p in paths.items():
        for wide in (False, True):
            back = HMatrix.load(p, wide=wide)
            assert back.meta["format"] == fmt
            for f in FIELDS:
                assert np.array_equal(getattr(back, f), getattr(hm, f)), (fmt, wide, f)
            if wide:
                assert back.a1.dtype == np.int64 and back.rowmat.dtype == np.float64
        assert np.array_equal(oracle_hmvm(HMatrix.load(p, wide=True), x), y0)


def _load64(path):
    lib = _lib.hmvm_lib()
    lv = _lib.Leaves64()
    fmt = C.c_int32(0)
    rc = lib.hmvm_b200_load_leaves64(path.encode(), C.byref(lv), C.byref(fmt))
    msg = lib.hmvm_b200_last_error().decode() if rc else ""
    if rc == 0:
        lib.hmvm_b200_free_leaves64(C.byref(lv))
        assert lv.nlf == 0 and not lv.rowmat  # cleared
    return rc, msg


def test_header_len_is_64_bit(hm, tmp_path):
    p = str(tmp_path / "h64.bin")
    hm.write_bin64(p)
    raw = bytearray(open(p, "rb").read())
    big = (1 << 33) + hm.len
    struct.pack_into("<q", raw, 16, big)
    open(p, "wb").write(raw)
    rc, msg = _load64(p)
    assert rc == _lib.HMVM_EFORMAT and str(big) in msg and str(hm.len) in msg


@pytest.mark.parametrize("fault", ["header_size", "truncated", "bad_marker", "ltmtx", "col_range", "neg_len",
                                   "bin2_false_saturation"])
def test_faults_return_status(hm, tmp_path, fault):
    """Host-side fault injection on the 64-bit loader: status codes, nothing leaked."""
    p = str(tmp_path / "bad.bin")
    hm.write_bin2(p) if fault == "bin2_false_saturation" else hm.write_bin64(p)
    raw = bytearray(open(p, "rb").read())
    if fault == "header_size":
        raw = struct.pack("<i", 24) + bytes(24) + struct.pack("<i", 24) + raw[28:]
    elif fault == "truncated":
        raw = raw[: len(raw) - 100]
    elif fault == "bad_marker":
        struct.pack_into("<i", raw, 24, 4 * hm.nlf + 4)  # ltmtx column's opening marker
    elif fault in ("ltmtx", "col_range"):
        col = 0 if fault == "ltmtx" else 4  # ltmtx, ndl, ndt, nstrtl, nstrtt, kt
        off = 28 + col * (4 * hm.nlf + 8) + 4
        struct.pack_into("<i", raw, off, 3 if fault == "ltmtx" else hm.nd)  # leaf 0
    elif fault == "neg_len":
        struct.pack_into("<q", raw, 16, -5)
    else:  # a bin2 len of INT32_MAX over a small file is not a saturated count
        struct.pack_into("<i", raw, 16, 2 ** 31 - 1)
    open(p, "wb").write(raw)
    rc, msg = _load64(p)
    assert rc == _lib.HMVM_EFORMAT, (rc, msg)


def test_missing_file():
    rc, msg = _load64("/nonexistent/h64.bin")
    assert rc == _lib.HMVM_EIO


# ---- beyond 2^31 elements (GPU) ---------------------------------------------

def _sparse_bin64(path, nd, blocks, kt):
    """A bin64 file of blocks x blocks low-rank leaves of rank kt tiling an
    nd x nd matrix, written with holes for the data (all zeros) except a few
    chosen entries.  Returns (leaf table, {(leaf, 'u'|'v', k, i): value}, element count)."""
    b = nd // blocks
    leaves = [(1, b, b, r * b + 1, c * b + 1, kt) for r in range(blocks) for c in range(blocks)]
    nlf = len(leaves)
    per_leaf = 2 * kt * b
    total = nlf * per_leaf
    # non-zeros: in the first and the last two leaves (the last one's offsets pass 2^31)
    rng = np.random.default_rng(9)
    picks = {}
    for leaf in (0, nlf - 1, nlf - 2):
        for k in rng.choice(kt, 3, replace=False):
            k = int(k)
            i_v, i_u = (int(v) for v in rng.integers(0, b, 2))
            picks[(leaf, "v", k, i_v)] = float(rng.integers(1, 8))
            picks[(leaf, "u", k, i_u)] = float(rng.integers(1, 8)) / 4
    with open(path, "wb") as f:
        def rec(payload):
            f.write(struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload)))
        rec(struct.pack("<3iq", nd, nlf, kt, total))
        for j in range(6):
            rec(np.array([lf[[0, 1, 2, 3, 4, 5][j]] for lf in leaves], np.int32).tobytes())
        nb = 8 * kt * b  # one factor record
        data_pos = []
        for _ in range(nlf):
            for _part in range(2):  # a1 = V [kt][ndt], a2 = U [kt][ndl]
                f.write(struct.pack("<i", nb))
                data_pos.append(f.tell())
                f.seek(nb, os.SEEK_CUR)
                f.write(struct.pack("<i", nb))
        for (leaf, part, k, i), val in picks.items():
            f.seek(data_pos[2 * leaf + (0 if part == "v" else 1)] + 8 * (i + k * b))
            f.write(struct.pack("<d", val))
    return leaves, picks, total


@pytest.mark.gpu
def test_beyond_int32_elements(gpu, tmp_path):
    psutil = pytest.importorskip("psutil")
    if psutil.virtual_memory().available < 96 * 2 ** 30:
        pytest.skip("needs ~40 GB of host memory for an 18.5 GB matrix and its plan")
    nd, blocks, kt = 65536, 4, 4400  # 2.31e9 elements: the last leaf's a1 and a2 pass 2^31
    path = str(tmp_path / "big.bin")
    leaves, picks, total = _sparse_bin64(path, nd, blocks, kt)
    assert total > 2 ** 31
    hm = HMatrix.load(path)
    assert hm.meta["format"] == 3 and hm.len == total and not hm.fits_matrix2()
    assert int(hm.a1[-1]) > 2 ** 31 and int(hm.a2[-1]) > 2 ** 31
    b = nd // blocks
    x = np.random.default_rng(4).integers(-4, 5, nd).astype(np.float64)
    want = np.zeros(nd)
    for leaf, (_, _, _, r0, c0, _) in enumerate(leaves):
        # y[r0-1+iu] += u[k][iu] * v[k][iv] * x[c0-1+iv], per rank-1 term k
        for (lf, part, k, iv), v in picks.items():
            if lf != leaf or part != "v":
                continue
            for (lf2, part2, k2, iu), u in picks.items():
                if lf2 == leaf and part2 == "u" and k2 == k:
                    want[r0 - 1 + iu] += u * v * x[c0 - 1 + iv]
    with Plan(hm, "fp64") as plan:
        y = plan.apply_host(x)
    del hm
    assert np.count_nonzero(want) > 0
    assert np.array_equal(y, want), relerr(y, want)
