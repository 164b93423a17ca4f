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
        assert v.stage1_teams <= 148 * 12 and v.stage2_teams <= 148 * 12  # kMultiWarpsPerSm (layout.hpp)
        tiles = np.ctypeslib.as_array((_lib.TileDesc * v.n_tiles).from_address(v.tiles))
        segs = np.ctypeslib.as_array((_lib.SegDesc * v.n_segs).from_address(v.segs))
        for td in tiles:
            zb = 0
            for sidx in range(int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])):
                ty, nc = seg_type(v, int(segs[sidx]["ncols"]))
                zb += -(-nc // SEG_VEC[ty]) * SEG_VEC[ty] * (8 if ty == 0 else 4)
            assert zb * nrhs_max <= (8192 if prec == 0 else 4096)  # kMultiZBytesF64, kMultiZBytes (layout.hpp)
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


# ---- the wide tensor-core layout (FP32 / mixed plans with nrhs_max >= 32) -------------
def _tcw_idesc(bf, n):
    """tcgen05 instruction descriptor, kind::f16, D FP32, A MN-major, B K-major, M 128."""
    return (1 << 4) | (bf << 7) | (bf << 10) | (1 << 15) | ((n >> 3) << 17) | ((128 >> 4) << 24)


def _tcw_program(view, tiles, segs, blocks):
    """The step program the kernel's producer walks is the segments' own
    grouping: per input group its src word, vector count, rows per K step, MMA
    counts per row block and last-group flag; per MMA (per segment, per block of
    its mask: hi x x_hi, hi x x_lo, and lo x x_hi for pairs; ordered by block)
    its first B row, A part, block, correction-accumulator flag (the correction
    products of row-stage blocks and of V-stage blocks of <= 64 rows), block rows
    and instruction descriptor; every B read stays inside its step."""
    ng, nops = view.n_tgroups, view.n_tops
    grp = np.ctypeslib.as_array(view.tgroups, (ng * 4,)).reshape(-1, 4).astype(np.int64)
    ops = np.ctypeslib.as_array(view.tops, ((nops + 12) * 2,)).reshape(-1, 2).astype(np.int64)
    first = np.ctypeslib.as_array(view.tgfirst, (view.n_tiles + 1,))
    assert np.all(ops[nops:] == 0)  # the zero templates the producer may read ahead
    gi, oi = 0, 0
    for k in range(view.n_tiles):
        assert first[k] == gi
        td = tiles[k]
        R = [(int(blocks[k]) >> (8 * b)) & 0xFF for b in range(4)]
        s, s1 = int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])
        while s < s1:
            g1 = s + 1
            while g1 < s1 and segs[g1]["src"] == segs[s]["src"] and \
                    (int(segs[g1]["ncols"]) & 0xFFFFFF) == (int(segs[s]["ncols"]) & 0xFFFFFF):
                g1 += 1
            nc = int(segs[s]["ncols"]) & 0xFFFFFF
            per_block, pre = [[], [], [], []], 0
            for z in range(s, g1):
                enc = int(segs[z]["ncols"])
                mask, pair = (enc >> 24) & 0xF, (enc >> 28) & 1
                for b in range(4):
                    if not mask >> b & 1:
                        continue
                    idesc = _tcw_idesc(view.tcw_bf16, max(16, (R[b] + 15) & ~15))
                    blk = (b << 13) | ((R[b] * 16) << 16)
                    corr = (1 << 15) if (k >= view.stage1_tiles or R[b] <= 64) else 0  # own accumulator
                    per_block[b] += [(pre | blk, idesc), (pre | (1 << 12) | blk | corr, idesc)]
                    if pair:
                        per_block[b].append(((pre + R[b]) | blk | corr, idesc))
                    pre += 2 * R[b] if pair else R[b]
            want = [t for b in range(4) for t in per_block[b]]  # each block's MMAs together
            counts = sum(len(per_block[b]) << (16 + 4 * b) for b in range(4))
            h = grp[gi]
            assert h[0] == int(segs[s]["src"]) & 0xFFFFFFFF and h[1] == (nc + 7) // 8
            assert h[2] == pre | ((1 << 12) if g1 == s1 else 0) | counts and h[3] == oi
            assert len(want) <= 12
            got = [tuple(int(v) for v in ops[oi + q]) for q in range(len(want))]
            assert got == want, (k, s, got, want)
            for t0, _ in want:  # the B rows of the MMA stay inside the group's rows of the step
                assert (t0 & 0xFFF) + ((t0 >> 16) // 16) <= pre
            gi, oi = gi + 1, oi + len(want)
            s = g1
    assert first[view.n_tiles] == gi == ng and oi == nops


def _tcw_bounds(view):
    """Every address hmvm_tcw_kernel and its helpers form stays inside its
    buffer, and every K step of an input group fits one 8 KiB ring chunk."""
    from hacapk_hmvm_b200 import _lib

    tiles = np.ctypeslib.as_array((_lib.TileDesc * view.n_tiles).from_address(view.tiles))
    segs = np.ctypeslib.as_array((_lib.SegDesc * view.n_segs).from_address(view.segs))
    blocks = np.ctypeslib.as_array(view.tblocks, (view.n_tiles,))
    covered = np.zeros(view.data_vectors, np.int32)
    for k in range(view.n_tiles):
        td = tiles[k]
        stage1 = k < view.stage1_tiles
        R = [(int(blocks[k]) >> (8 * b)) & 0xFF for b in range(4)]
        nblk = sum(1 for r in R if r)
        assert R[:nblk] == [r for r in R if r] and all(r <= (128 if stage1 else 32) for r in R)
        assert nblk <= (2 if stage1 else 4)  # the kernel's TMEM geometry per stage
        assert int(td["nrows"]) == sum(R) >= 1
        off, nrec = int(td["data_off"]), int(td["nvec"])
        assert 0 <= off and off + nrec <= view.data_vectors
        covered[off:off + nrec] += 1
        tot, used = 0, 0
        s0, s1 = int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])
        s = s0
        while s < s1:
            g1 = s + 1
            while g1 < s1 and segs[g1]["src"] == segs[s]["src"] and \
                    (int(segs[g1]["ncols"]) & 0xFFFFFF) == (int(segs[s]["ncols"]) & 0xFFFFFF):
                g1 += 1
            nc = int(segs[s]["ncols"]) & 0xFFFFFF
            step = 0  # bytes of a full K step of the group
            for z in range(s, g1):
                src, enc = int(segs[z]["src"]), int(segs[z]["ncols"])
                mask, fmt = (enc >> 24) & 0xF, (enc >> 28) & 1
                assert enc >> 29 == 0 and mask and all(R[b] for b in range(4) if mask >> b & 1)
                used |= mask
                rows = sum(R[b] for b in range(4) if mask >> b & 1)
                step += 2 * rows * 16 * (2 if fmt else 1)
                tot += -(-nc // 8) * (2 if fmt else 1) * rows
                if src < 0:
                    assert not stage1 and (src & 0x7FFFFFFF) + nc <= view.t_len
                else:
                    assert src + nc <= view.nd
            jobs = sum(bin((int(segs[z]["ncols"]) >> 24) & 0xF).count("1") for z in range(s, g1))
            assert step <= 8192 and jobs <= 4  # a chunk, and the kernel's 4 MMA jobs per input group
            s = g1
        assert tot == nrec
        assert (int(td["mode"]) >> 4) == used
        pad, nrows = int(td["_pad"]), int(td["nrows"])
        mode = int(td["mode"]) & 3
        if stage1:
            assert mode in (1, 2) and pad + nrows <= view.tscale_rows0
            assert int(td["out_base"]) + nrows <= (view.tscale_rows0 if mode == 1 else view.p_len)
        else:
            assert mode == 0 and view.tscale_rows0 <= pad and pad + nrows <= view.n_tscale
            assert int(td["out_base"]) + nrows <= view.nd
    assert np.all(covered == 1)  # the items partition the stream
    _tcw_program(view, tiles, segs, blocks)
    n1 = view.tscale_rows0
    out_idx = np.ctypeslib.as_array(view.out_idx, (n1,)) if n1 else np.zeros(0, np.int32)
    assert np.all((out_idx >= 0) & (out_idx < max(view.t_len, 1)))
    if view.n_red1:
        red = np.ctypeslib.as_array(view.red1, (view.n_red1 * 4,)).reshape(-1, 4)
        assert np.all(red[:, 0] < view.t_len)
        assert np.all(red[:, 1] + (red[:, 2] - 1) * red[:, 3] < view.p_len)
    sc = np.ctypeslib.as_array(view.tscale, (view.n_tscale,))
    assert np.all(np.isfinite(sc)) and np.all(sc > 0)
    assert np.all(np.log2(sc) == np.round(np.log2(sc)))  # powers of two: exact scaling


@pytest.mark.parametrize("prec,fmt,tol", [(2, "fp16", 1e-4), (2, "bf16", 1e-4), (1, None, 1e-5)])
@pytest.mark.parametrize("case", [(3000, "sphere", 3), (2500, "plate", 4), (2200, "cube", 6)],
                         ids=lambda c: f"{c[1]}{c[0]}")
def test_tcw_layout_against_oracle(prec, fmt, tol, case):
    from helpers import emulate_tcw

    n, geo, seed = case
    hm = HMatrix.generate(n, geo, eta=2.0, eps=1e-4, leaf_size=32, seed=seed)
    kw = dict(precision=prec, nrhs_max=128, num_sms=16)
    if fmt:
        kw["mixed_lr_format"] = fmt
    h, view = layout_for(hm, **kw)
    assert view.tcw == 1 and view.tcw_bf16 == (fmt == "bf16")
    _tcw_bounds(view)
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (3, hm.nd)) * np.array([1.0, 1e-9, 1e7])[:, None]
    Y = emulate_tcw(view, X)
    for r in range(3):
        assert relerr(Y[r], oracle_hmvm(hm, X[r])) <= tol, (r, relerr(Y[r], oracle_hmvm(hm, X[r])))


def test_tcw_layout_split_panels():
    """Large V-stage panels are cut into K-step ranges whose partial sums the
    reduction adds; the result is unchanged."""
    from helpers import emulate_tcw

    hm = HMatrix.generate(12000, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=8)
    h, view = layout_for(hm, precision=1, nrhs_max=128, num_sms=148)
    assert view.n_red1 > 0
    _tcw_bounds(view)
    X = np.random.default_rng(3).standard_normal((2, hm.nd))
    Y = emulate_tcw(view, X)
    for r in range(2):
        assert relerr(Y[r], oracle_hmvm(hm, X[r])) <= 1e-5
