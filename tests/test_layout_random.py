"""The host planner on random leaf lists, checked without a GPU.

Generated H-matrices are well-formed partitions; the reference's HMVM
(`src_hmvm/src_cpp/hmvm_seq.cpp:154-227`) only needs each leaf's ranges and
offsets to be in bounds.  These tables have ragged sizes, empty leaves
(kt = 0, ndl = 0 or ndt = 0), overlapping blocks (their products add up) and
rows no leaf covers, and every layout is checked for in-bounds addressing
and for a CPU walk of its repacked data that reproduces the oracle."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import emulate_layout, layout_for, oracle_hmvm
from layout_checks import check_layout_bounds
from test_layout import MIXED_DEFAULT_CFGS, MIXED_ZBYTES


@st.composite
def leaf_tables(draw):
    nd = draw(st.integers(1, 300))
    nlf = draw(st.integers(0, 40))
    seed = draw(st.integers(0, 2**31 - 1))
    rng = np.random.default_rng(seed)
    cols = {k: [] for k in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2")}
    data, off = [], 0

    def extent(start):
        # 0 with a small probability, else 1 .. what is left of 1..nd
        return 0 if rng.random() < 0.05 else int(rng.integers(1, nd - start + 2))

    for _ in range(nlf):
        sl, stt = int(rng.integers(1, nd + 1)), int(rng.integers(1, nd + 1))
        ndl, ndt = extent(sl), extent(stt)
        lr = rng.random() < 0.5
        kt = int(rng.integers(0, 12)) if lr else 0
        if lr:
            a1, a2 = off, off + kt * ndt
            n = kt * (ndl + ndt)
        else:
            a1 = a2 = off
            n = ndl * ndt
        for k, v in zip(cols, (1 if lr else 2, kt, ndl, ndt, sl, stt, a1, a2)):
            cols[k].append(v)
        data.append(rng.standard_normal(n))
        off += n
    rowmat = np.concatenate(data) if data else np.zeros(0)
    ktmax = max(cols["kt"], default=0)
    hm = HMatrix.from_arrays(nd, ktmax, cols["ltmtx"], cols["kt"], cols["ndl"], cols["ndt"], cols["nstrtl"],
                             cols["nstrtt"], cols["a1"], cols["a2"], rowmat)
    return hm, rng.uniform(-1, 1, nd)


PLAIN_OPTS = [dict(), dict(kernel=0), dict(split_cols=2), dict(max_tile_rows=3), dict(nrhs_max=8),
              dict(stage1_cfg=3, stage2_cfg=5, num_sms=2)]
MIXED_OPTS = [dict(), dict(mixed_lr_format="bf16", split_cols=8), dict(max_tile_rows=5, num_sms=3),
              dict(stage1_cfg=5, stage2_cfg=1), dict(nrhs_max=16)]


def _abs_bound(hm, x):
    """(|U| |V^T| + |D|) |x| row by row: the scale a row's rounding errors are
    measured against, since a row whose terms cancel has no relative accuracy
    to keep."""
    ha = HMatrix.from_arrays(hm.nd, hm.ktmax, hm.ltmtx, hm.kt, hm.ndl, hm.ndt, hm.nstrtl, hm.nstrtt, hm.a1,
                             hm.a2, np.abs(hm.rowmat.astype(np.float64)))
    return oracle_hmvm(ha, np.abs(x))


def _check(hm, x, prec, opts, tol):
    """Bounds of the layout, then |y - y_oracle| <= tol * (|H| |x|) per row."""
    h, v = layout_for(hm, precision=prec, **opts)
    try:
        if prec == 2:
            check_layout_bounds(v, zbytes=(MIXED_ZBYTES[opts.get("stage1_cfg", MIXED_DEFAULT_CFGS[0])],
                                           MIXED_ZBYTES[opts.get("stage2_cfg", MIXED_DEFAULT_CFGS[1])]))
        else:
            check_layout_bounds(v)
        y, yo = emulate_layout(v, x), oracle_hmvm(hm, x)
        bound = tol * _abs_bound(hm, x)
        bad = np.abs(y - yo) > bound
        assert not bad.any(), (prec, opts, np.flatnonzero(bad)[:5], (y - yo)[bad][:5], bound[bad][:5])
    finally:
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


@settings(max_examples=40, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(leaf_tables())
def test_random_tables_plain(table):
    hm, x = table
    for opts in PLAIN_OPTS:
        _check(hm, x, 0, opts, 1e-13)
    hf = hm.to_float()
    for opts in PLAIN_OPTS[:3]:
        _check(hf, x, 1, opts, 1e-5)


@settings(max_examples=25, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(leaf_tables())
def test_random_tables_mixed(table):
    """Mixed plans store random factors in 16-bit and FP8 formats, so the walk
    only has to match the oracle to the formats' precision (FP16 columns:
    2^-11 per element, E4M3 only below 1e-4 of a block): any addressing mistake
    would be O(1)."""
    hm, x = table
    for opts in MIXED_OPTS:
        _check(hm, x, 2, opts, 2e-3)


@pytest.mark.parametrize("nd", [1, 33, 257])
def test_every_row_covered_twice(nd):
    """Two full dense leaves over the same block: every y row is their sum."""
    rng = np.random.default_rng(nd)
    a = rng.standard_normal(nd * nd)
    b = rng.standard_normal(nd * nd)
    hm = HMatrix.from_arrays(nd, 0, [2, 2], [0, 0], [nd, nd], [nd, nd], [1, 1], [1, 1], [0, nd * nd],
                             [0, nd * nd], np.concatenate([a, b]))
    x = rng.uniform(-1, 1, nd)
    for opts in PLAIN_OPTS:
        _check(hm, x, 0, opts, 1e-13)
