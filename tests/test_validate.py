"""Descriptor bounds checks (csrc/validate.hpp, hmvm_b200_layout_validate):
every layout the planner builds passes them, and a layout with one
descriptor pointed outside its buffer is rejected with a message naming it.
The same checks run on the device in the HMVM_DEVICE_CHECKS build
(tests/test_device_checks_gpu.py)."""
import ctypes as C
import os

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import layout_for

OPTS = [
    dict(precision=0), dict(precision=1), dict(precision=0, kernel=0), dict(precision=0, split_cols=8),
    dict(precision=1, max_tile_rows=7), dict(precision=2), dict(precision=2, mixed_lr_format="bf16"),
    dict(precision=2, stage1_cfg=9, stage2_cfg=6), dict(precision=0, nrhs_max=8), dict(precision=1, nrhs_max=4),
    dict(precision=2, nrhs_max=2), dict(precision=2, nrhs_max=16),
]


def _validate(h):
    return _lib.hmvm_lib().hmvm_b200_layout_validate(h)


def _msg():
    return _lib.hmvm_lib().hmvm_b200_last_error().decode(errors="replace")


@pytest.mark.parametrize("case", [(1500, "sphere", 2.0, 1e-4, 32), (900, "plate", 2.0, 1e-3, 8),
                                  (777, "cube", 1.0, 1e-4, 45)], ids=lambda c: f"{c[1]}{c[0]}")
def test_planned_layouts_pass(case):
    n, geo, eta, eps, leaf = case
    hm = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=5)
    for opts in OPTS:
        h, v = layout_for(hm, **opts)
        try:
            assert _validate(h) == _lib.HMVM_OK, (opts, _msg())
        finally:
            _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def _arrays(v):
    tiles = np.ctypeslib.as_array((_lib.TileDesc * v.n_tiles).from_address(v.tiles))
    segs = np.ctypeslib.as_array((_lib.SegDesc * v.n_segs).from_address(v.segs))
    return tiles, segs


def _corruptions(v, tiles, segs):
    """(what, phrase, apply) triples; apply changes one field in place and
    returns a function that restores it."""
    s1 = int(v.stage1_tiles)
    row2 = s1  # the first row-stage item: y rows (mode 0) or partial sums (mode 2)
    out_end = v.nd if tiles[row2]["mode"] == 0 else v.p_len
    slot1 = next((k for k in range(s1) if tiles[k]["mode"] == 1), None)
    xseg = next(j for j in range(v.n_segs) if segs[j]["src"] >= 0)
    tb2 = np.ctypeslib.as_array(v.team_begin2, (v.stage2_teams + 1,))

    def setter(arr, idx, field, value):
        def apply():
            old = arr[idx][field] if field else arr[idx]
            if field:
                arr[idx][field] = value
            else:
                arr[idx] = value
            def restore():
                if field:
                    arr[idx][field] = old
                else:
                    arr[idx] = old
            return restore
        return apply

    out = [
        ("data range", "leave the data stream", setter(tiles, row2, "data_off", v.data_vectors)),
        ("segment range", "segment descriptors", setter(tiles, row2, "seg_begin", v.n_segs)),
        ("no rows", "rows are outside", setter(tiles, row2, "nrows", 0)),
        ("33 rows", "rows are outside", setter(tiles, row2, "nrows", 33)),
        ("output row", "output rows", setter(tiles, row2, "out_base", out_end)),
        ("x column", "columns leave x or t", setter(segs, xseg, "src", v.nd)),
        ("team ranges", "team ranges", setter(tb2, v.stage2_teams, None, int(tb2[v.stage2_teams]) - 1)),
    ]
    if slot1 is not None:
        out_idx = np.ctypeslib.as_array(v.out_idx, (int(tiles[slot1]["out_base"]) + 1,))
        out.append(("t slot", "t slot", setter(out_idx, int(tiles[slot1]["out_base"]), None, v.t_len)))
    return out


@pytest.mark.parametrize("prec", [0, 2], ids=["fp64", "mixed"])
def test_corrupted_descriptor_rejected(prec):
    hm = HMatrix.generate(1500, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=5)
    h, v = layout_for(hm, precision=prec)
    try:
        tiles, segs = _arrays(v)
        assert _validate(h) == _lib.HMVM_OK
        for what, phrase, apply in _corruptions(v, tiles, segs):
            restore = apply()
            try:
                assert _validate(h) == _lib.HMVM_ERANGE, what
                assert phrase in _msg(), (what, _msg())
            finally:
                restore()
            assert _validate(h) == _lib.HMVM_OK, what
        # a reduction entry whose parts run past the partial sums
        if v.n_red2 > 0:
            red = np.ctypeslib.as_array(v.red2, (v.n_red2 * 4,))
            old = int(red[2])
            red[2] = 1 << 20
            try:
                assert _validate(h) == _lib.HMVM_ERANGE and "reduction entry" in _msg()
            finally:
                red[2] = old
    finally:
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def test_checked_library_exports_the_same_symbols():
    """The HMVM_DEVICE_CHECKS build exports every entry point of the header."""
    from hacapk_hmvm_b200 import build

    if not os.path.exists(build.LIB_HMVM_CHECKED):
        pytest.skip("the checked library is built by build_all()")
    lib = C.CDLL(build.LIB_HMVM_CHECKED)
    for name in _lib.HMVM_SIGNATURES:
        assert hasattr(lib, name), name
