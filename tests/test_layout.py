"""The host planner (csrc/layout.cpp), checked without a GPU: every address the
kernels form stays inside its buffer, every row is written exactly once, and a
CPU walk of the repacked layout reproduces the oracle."""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import emulate_layout, layout_for, oracle_hmvm, relerr
from layout_checks import check_layout_bounds

CASES = [(1500, "sphere", 2.0, 1e-4, 32), (1200, "cube", 1.0, 1e-6, 16), (900, "plate", 2.0, 1e-3, 8),
         (777, "cube", 1.0, 1e-4, 45)]
OPTS = [dict(), dict(kernel=0), dict(split_cols=2), dict(split_cols=40), dict(max_tile_rows=7),
        dict(kernel=0, stage1_cfg=0, stage2_cfg=7, ctas_per_sm=1), dict(stage1_cfg=3, stage2_cfg=1, ctas_per_sm=1),
        dict(stage1_cfg=5, stage2_cfg=4)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[1]}{c[0]}")
def test_layout_bounds_and_emulation(case):
    n, geo, eta, eps, leaf = case
    hm = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=5)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    yo = oracle_hmvm(hm, x)
    for prec in (0, 1):
        for opts in OPTS:
            h, v = layout_for(hm, precision=prec, **opts)
            check_layout_bounds(v)
            err = relerr(emulate_layout(v, x), yo)
            assert err < (1e-14 if prec == 0 else 1e-6), (prec, opts, err)
            _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


MIXED_ZBYTES = {0: 2048, 1: 4096, 2: 4096, 3: 4096, 4: 4096, 5: 2048, 6: 2048, 7: 2048, 8: 4096, 9: 2048, 10: 2048}  # kMixedCfgs (layout.hpp)
MIXED_DEFAULT_CFGS = (10, 8)  # kDefaultMixedCfg1, kDefaultMixedCfg2 (layout.hpp)
MIXED_OPTS = [dict(), dict(mixed_lr_format="bf16"), dict(mixed_fp8_eps=0.0), dict(mixed_fp32_tau=2.0),
              dict(split_cols=8), dict(max_tile_rows=5), dict(stage1_cfg=5, stage2_cfg=1, ctas_per_sm=1),
              dict(stage1_cfg=7, stage2_cfg=4), dict(stage1_cfg=9, stage2_cfg=10)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[1]}{c[0]}")
def test_mixed_layout_bounds_and_emulation(case):
    """Mixed plans: bounds, the per-item input buffer, and the decoded formats
    give relerr <= 1e-4 against the FP64 oracle."""
    n, geo, eta, eps, leaf = case
    hm = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=5)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    yo = oracle_hmvm(hm, x)
    for opts in MIXED_OPTS:
        h, v = layout_for(hm, precision=2, **opts)
        check_layout_bounds(v, zbytes=(MIXED_ZBYTES[opts.get("stage1_cfg", MIXED_DEFAULT_CFGS[0])],
                                       MIXED_ZBYTES[opts.get("stage2_cfg", MIXED_DEFAULT_CFGS[1])]))
        err = relerr(emulate_layout(v, x), yo)
        assert err < 1e-4, (opts, err)
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def test_mixed_column_classes():
    """Columns at or above tau*|block| are FP32, below eps*|block| FP8, the
    rest FP16; the stage-1 rows carry scale s_u*s_v."""
    from helpers import decode_vectors

    hm = HMatrix.generate(1500, "sphere", eps=1e-6, leaf_size=24, seed=3)
    h, v = layout_for(hm, precision=2)
    segs = np.ctypeslib.as_array((_lib.SegDesc * v.n_segs).from_address(v.segs))
    types = segs["ncols"].astype(np.int64) >> 28
    assert set(np.unique(types)) <= {0, 1, 2, 3}
    assert (types == 3).any() and (types == 2).any() and (types == 1).any() and (types == 0).any()
    assert np.all(np.ctypeslib.as_array(v.rowscale, (v.n_rowscale,)) > 0)
    _lib.hmvm_lib().hmvm_b200_layout_destroy(h)
    # the FP8 share grows with the threshold, the FP32 share with 1/tau
    def counts(**o):
        h, v = layout_for(hm, precision=2, **o)
        segs = np.ctypeslib.as_array((_lib.SegDesc * v.n_segs).from_address(v.segs))
        ty, nc = segs["ncols"].astype(np.int64) >> 28, segs["ncols"].astype(np.int64) & 0x0FFFFFFF
        tiles = np.ctypeslib.as_array((_lib.TileDesc * v.n_tiles).from_address(v.tiles))
        first = tiles[:v.stage1_tiles]["seg_begin"]
        rows = tiles[:v.stage1_tiles]["nrows"]
        out = {t: int(rows[ty[first] == t].sum()) for t in (1, 2, 3)}
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)
        return out
    a, b = counts(mixed_fp8_eps=1e-5), counts(mixed_fp8_eps=1e-3)
    assert b[3] > a[3]
    c, d = counts(mixed_fp32_tau=0.9), counts(mixed_fp32_tau=0.1)
    assert d[1] > c[1]
    assert counts(mixed_fp8_eps=0.0)[3] == 0


@pytest.mark.parametrize("nrhs_max", [2, 4, 8])
def test_multi_rhs_items_fit_input_buffer(nrhs_max):
    """Plans for the multi-RHS kernel: every item's inputs for nrhs_max
    right-hand sides fit its 8 KiB buffer, and the teams are the multi-RHS
    kernel's (8 per SM)."""
    from layout_checks import SEG_VEC, seg_type

    hm = HMatrix.generate(2500, "cube", eps=1e-6, leaf_size=24, seed=4)
    x = np.random.default_rng(3).uniform(-1, 1, hm.nd)
    yo = oracle_hmvm(hm, x)
    for prec in (0, 1, 2):
        h, v = layout_for(hm, precision=prec, nrhs_max=nrhs_max)
        check_layout_bounds(v)
        assert v.stage1_teams <= 148 * 8 and v.stage2_teams <= 148 * 8
        tiles = np.ctypeslib.as_array((_lib.TileDesc * v.n_tiles).from_address(v.tiles))
        segs = np.ctypeslib.as_array((_lib.SegDesc * v.n_segs).from_address(v.segs))
        for td in tiles:
            zb = 0
            for sidx in range(int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])):
                ty, nc = seg_type(v, int(segs[sidx]["ncols"]))
                zb += -(-nc // SEG_VEC[ty]) * SEG_VEC[ty] * (8 if ty == 0 else 4)
            assert zb * nrhs_max <= 8192
        assert relerr(emulate_layout(v, x), yo) < (1e-14 if prec == 0 else 1e-6 if prec == 1 else 1e-4)
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def test_stream_items_fit_input_buffer():
    from hacapk_hmvm_b200._lib import TileDesc

    hm = HMatrix.generate(3000, "sphere", seed=2)
    zcap = {0: 256, 1: 512, 2: 256, 3: 128, 4: 512, 5: 256, 6: 256, 7: 512}  # kStreamCfgs (layout.hpp)
    for cfg in range(8):
        for prec, vec in ((0, 2), (1, 4)):
            h, v = layout_for(hm, precision=prec, stage1_cfg=cfg, stage2_cfg=cfg)
            tiles = np.ctypeslib.as_array((TileDesc * v.n_tiles).from_address(v.tiles))
            assert (tiles["nvec"].astype(np.int64) * vec).max() <= zcap[cfg]
            _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def test_invalid_leaf_tables_rejected():
    import ctypes as C

    good = HMatrix.from_arrays(4, 1, [1, 2], [1, 0], [2, 2], [2, 4], [1, 3], [3, 1], [0, 4], [2, 0],
                               np.arange(1.0, 13.0))
    lib = _lib.hmvm_lib()
    h, v = layout_for(good)
    lib.hmvm_b200_layout_destroy(h)
    bad_cases = {"ltmtx": ("ltmtx", 0, 3), "kt": ("kt", 0, 2), "rows": ("nstrtl", 1, 4),
                 "cols": ("nstrtt", 0, 4), "a1": ("a1", 1, 10)}
    for name, (field, i, val) in bad_cases.items():
        bad = HMatrix.from_arrays(good.nd, good.ktmax, good.ltmtx, good.kt, good.ndl, good.ndt, good.nstrtl,
                                  good.nstrtt, good.a1, good.a2, good.rowmat)
        getattr(bad, field)[i] = val
        with pytest.raises(_lib.HMVMError) as e:
            layout_for(bad)
        assert e.value.status == _lib.HMVM_EINVAL, name
