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


def test_stream_items_fit_input_buffer():
    from hacapk_hmvm_b200._lib import TileDesc

    hm = HMatrix.generate(3000, "sphere", seed=2)
    zcap = {0: 256, 1: 512, 2: 256, 3: 128, 4: 512, 5: 256}  # kStreamCfgs (layout.hpp)
    for cfg in range(6):
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
