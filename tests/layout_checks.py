"""Bounds checks of a layout: every address the kernels form stays inside its buffer."""
import ctypes as C

import numpy as np


SEG_VEC = {0: 2, 1: 4, 2: 8, 3: 16, 4: 8}  # elements per 16-byte vector by storage type


def seg_type(view, enc):
    """(storage type, columns) of a segment descriptor's ncols field."""
    if view.precision == 2:
        return enc >> 28, enc & 0x0FFFFFFF
    return (0 if view.precision == 0 else 1), enc


def check_layout_bounds(view, zbytes=None):
    """zbytes: (mixed plans) the kernels' input buffers per item, in bytes,
    as (V stage, row stage)."""
    from hacapk_hmvm_b200 import _lib

    mixed = view.precision == 2
    VEC = view.vec
    nt = view.n_tiles
    tiles = np.ctypeslib.as_array((_lib.TileDesc * nt).from_address(view.tiles)) if nt else None
    segs = np.ctypeslib.as_array((_lib.SegDesc * view.n_segs).from_address(view.segs)) if view.n_segs else None
    tb1 = np.ctypeslib.as_array(view.team_begin1, (view.stage1_teams + 1,))
    tb2 = np.ctypeslib.as_array(view.team_begin2, (view.stage2_teams + 1,))
    assert tb1[0] == 0 and tb1[-1] == view.stage1_tiles and np.all(np.diff(tb1) >= 0)
    assert tb2[0] == view.stage1_tiles and tb2[-1] == nt and np.all(np.diff(tb2) >= 0)
    n_out = 0
    covered = np.zeros(view.nd, np.int32)
    for k in range(nt):
        td = tiles[k]
        R, nvec, off = int(td["nrows"]), int(td["nvec"]), int(td["data_off"])
        assert 1 <= R <= 32 and nvec >= 0
        assert 0 <= off and off + nvec * R <= view.data_vectors
        s0, ns = int(td["seg_begin"]), int(td["nseg"])
        assert 0 <= s0 and s0 + ns <= view.n_segs
        tot = zb = 0
        if mixed:
            assert ns <= 32
            assert k >= view.stage1_tiles or ns == 1  # the V-stage kernel runs one segment per item
        for s in range(s0, s0 + ns):
            src = int(segs[s]["src"])
            ty, ncols = seg_type(view, int(segs[s]["ncols"]))
            vs = SEG_VEC[ty]
            assert ncols >= 1 and ty in SEG_VEC
            if src < 0:
                slot = src & 0x7FFFFFFF
                if mixed:  # t is FP32; the kernel reads exactly ncols slots
                    assert ty != 0 and slot + ncols <= view.t_len
                else:
                    assert slot % VEC == 0
                    assert slot + -(-ncols // VEC) * VEC <= view.t_len
            else:
                assert 0 <= src and src + ncols <= view.nd
            tot += -(-ncols // vs)
            zb += -(-ncols // vs) * vs * (8 if ty == 0 else 4)
        assert tot == nvec
        if mixed and zbytes is not None:
            assert zb <= zbytes[0 if k < view.stage1_tiles else 1]
        if mixed and k < view.stage1_tiles:
            assert 0 <= int(td["_pad"]) and int(td["_pad"]) + R <= view.n_rowscale
        ob, mode = int(td["out_base"]), int(td["mode"])
        if k < view.stage1_tiles:
            assert mode in (1, 2)
            if mode == 2:
                assert 0 <= ob and ob + R <= view.p_len
            else:
                n_out = max(n_out, ob + R)
        else:
            assert mode in (0, 2)
            if mode == 0:
                assert 0 <= ob and ob + R <= view.nd
                covered[ob:ob + R] += 1
            else:
                assert 0 <= ob and ob + R <= view.p_len
    if n_out:
        out_idx = np.ctypeslib.as_array(view.out_idx, (n_out,))
        assert np.all((out_idx >= 0) & (out_idx < view.t_len))
        assert len(np.unique(out_idx)) == len(out_idx)
    if view.n_red1:
        red = np.ctypeslib.as_array(view.red1, (view.n_red1 * 4,)).reshape(-1, 4)
        assert np.all((red[:, 0] >= 0) & (red[:, 0] < view.t_len))
        assert np.all(red[:, 1] >= 0) and np.all(red[:, 1] + (red[:, 2] - 1) * red[:, 3] < view.p_len)
    if view.n_red2:
        red = np.ctypeslib.as_array(view.red2, (view.n_red2 * 4,)).reshape(-1, 4)
        assert np.all((red[:, 0] >= 0) & (red[:, 0] < view.nd))
        assert np.all(red[:, 1] >= 0) and np.all(red[:, 1] + (red[:, 2] - 1) * red[:, 3] < view.p_len)
        covered[red[:, 0]] += 1
    assert np.all(covered == 1), "every row must be written exactly once (by a tile or a reduction)"
    # the items of one team form one contiguous region of the data stream
    for tbeg in (tb1, tb2):
        for a, b in zip(tbeg[:-1], tbeg[1:]):
            for k in range(a + 1, b):
                prev = tiles[k - 1]
                assert int(tiles[k]["data_off"]) == int(prev["data_off"]) + int(prev["nvec"]) * int(prev["nrows"])
