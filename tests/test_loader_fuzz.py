"""The loaders on damaged files: a truncated file or any int32 of a record
overwritten (record markers, counts, leaf headers, offsets) must give a status
code, or a table that the planner accepts and walks in bounds -- never a crash
or a read past the file.  The reference's loaders (src_hmvm/src_cpp/
loadmatrix.cpp:7-250) trust every field; the library's replace them at the
boundary where files come from outside."""
import ctypes as C
import os

import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import GOLDEN
from layout_checks import check_layout_bounds

OK_OR_FORMAT = (_lib.HMVM_OK, _lib.HMVM_EFORMAT, _lib.HMVM_EIO)
SRC = os.path.join(GOLDEN, "kat6_hmatrix_1.bin")
SRC_BIG = os.path.join(GOLDEN, "plate200_hmatrix_1.bin")


def _variants(tmp):
    """The same matrix as hmatrix_1.bin, hmatrix_2.bin and the 64-bit variant."""
    out = {}
    for name, src in (("kat", SRC), ("plate", SRC_BIG)):
        hm = HMatrix.load(src)
        p2, p3 = os.path.join(tmp, f"{name}_2.bin"), os.path.join(tmp, f"{name}_64.bin")
        hm.write_bin2(p2)
        hm.write_bin64(p3)
        out[(name, 1)] = open(src, "rb").read()
        out[(name, 2)] = open(p2, "rb").read()
        out[(name, 3)] = open(p3, "rb").read()
    return out


@pytest.fixture(scope="module")
def variants(tmp_path_factory):
    return _variants(str(tmp_path_factory.mktemp("fuzz")))


INTERESTING = [0, 1, -1, 2, 3, 6, 7, 8, 12, 16, 20, 199, 200, 201, 2**31 - 1, -2**31, 2**30, 65536]


def _mutate(raw, data):
    """Truncate, or overwrite one to three int32 words in the first 4 KB (the
    headers, markers and the leading leaf records)."""
    buf = bytearray(raw)
    if data.draw(st.booleans(), label="truncate") and len(buf) > 1:
        return bytes(buf[: data.draw(st.integers(0, len(buf) - 1), label="cut")])
    words = min(len(buf), 4096) // 4
    for _ in range(data.draw(st.integers(1, 3), label="edits")):
        w = data.draw(st.integers(0, words - 1), label="word")
        v = data.draw(st.one_of(st.sampled_from(INTERESTING), st.integers(-2**31, 2**31 - 1)), label="value")
        buf[4 * w: 4 * w + 4] = int(v).to_bytes(4, "little", signed=True)
    return bytes(buf)


def _check_loaded_leaves(lv):
    """An accepted table must plan and address only inside its buffers.  An
    edited nd can make a valid table of up to 2^31 - 1 rows with the same few
    leaves; the planner writes every row (uncovered rows are zero), so its time
    grows with nd: it runs here up to 10^7 rows, the row-by-row Python walk up
    to 10^6."""
    if lv.nd > 10**7:
        return
    lib = _lib.hmvm_lib()
    o = _lib.PlanOpts()
    lib.hmvm_b200_default_opts(C.byref(o))
    h = C.c_void_p()
    rc = lib.hmvm_b200_layout_build64(C.byref(lv), 0, C.byref(o), 148, C.byref(h))
    assert rc == _lib.HMVM_OK, lib.hmvm_b200_last_error()
    v = _lib.LayoutView()
    _lib.check(lib.hmvm_b200_layout_view(h, C.byref(v)), "layout view")
    if lv.nd <= 10**6:
        check_layout_bounds(v)
    lib.hmvm_b200_layout_destroy(h)


@settings(max_examples=150, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.function_scoped_fixture])
@given(data=st.data())
def test_damaged_files_give_status_or_valid_table(variants, tmp_path, data):
    lib = _lib.hmvm_lib()
    key = data.draw(st.sampled_from(sorted(variants)), label="file")
    raw = _mutate(variants[key], data)
    p = str(tmp_path / "damaged.bin")
    with open(p, "wb") as f:
        f.write(raw)
    fmt = key[1]
    if fmt == 1:
        m1, m2 = _lib.Matrix_d(), _lib.Matrix2_d()
        rc = lib.hmvm_b200_load_hmatrix(p.encode(), C.byref(m1), C.byref(m2))
        assert rc in OK_OR_FORMAT, rc
        if rc == _lib.HMVM_OK:
            lib.hmvm_b200_free_matrix_d(C.byref(m1))
            lib.hmvm_b200_free_matrix2_d(C.byref(m2))
        else:
            assert not m2.rowmat
    elif fmt == 2:
        m2 = _lib.Matrix2_d()
        rc = lib.hmvm_b200_load_hmatrix2(p.encode(), C.byref(m2))
        assert rc in OK_OR_FORMAT, rc
        if rc == _lib.HMVM_OK:
            lib.hmvm_b200_free_matrix2_d(C.byref(m2))
        else:
            assert not m2.rowmat
    lv, got = _lib.Leaves64(), C.c_int32(0)
    rc = lib.hmvm_b200_load_leaves64(p.encode(), C.byref(lv), C.byref(got))
    assert rc in OK_OR_FORMAT, rc
    if rc == _lib.HMVM_OK:
        try:
            _check_loaded_leaves(lv)
        finally:
            lib.hmvm_b200_free_leaves64(C.byref(lv))
