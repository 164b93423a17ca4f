"""Test helpers: ctypes access to the oracles and a CPU emulation of the
repacked layout.

The oracles are test infrastructure (oracle/): liboracle.so is the plain-C
restatement of the reference HMVM, oracle/_ref/libhmvm_ref.so is the
reference's own code built from its sources.  Only tests, the smoke check and
bench.py's CPU-baseline leg use them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libhmvm_ref.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")
# Where the reference's source tree lies (its sample mesh and matrix and its
# headers are read from there; tests that need them are skipped when it is
# absent).  Override with the HACAPK_REFERENCE environment variable.
REFERENCE = os.environ.get("HACAPK_REFERENCE", "/root/reference")
SAMPLE_BIN = os.path.join(REFERENCE, "src_hdump", "hmatrix_sample.bin")
SAMPLE_PBF = os.path.join(REFERENCE, "src_hdump", "input_sample.pbf")
REF_INC = os.path.join(REFERENCE, "src_hmvm", "src_cpp")

_P = C.c_void_p


def _p(a):
    return a.ctypes.data_as(_P)


_orc = None
_ref = None


def oracle_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            raise FileNotFoundError(f"{ORACLE_SO} missing: run `make -C oracle`")
        lib = C.CDLL(ORACLE_SO)
        lib.orc_open.restype = C.c_void_p
        lib.orc_open.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int)]
        lib.orc_close.argtypes = [C.c_void_p]
        lib.orc_info.argtypes = [C.c_void_p, _P]
        lib.orc_export.argtypes = [C.c_void_p] + [_P] * 9
        for fn in ("orc_hmvm_seq2_d", "orc_hmvm_seq2_f"):
            getattr(lib, fn).argtypes = [C.c_int32, C.c_int32, C.c_int32] + [_P] * 11 + [C.c_int]
        lib.orc_omp2_d.argtypes = [C.c_int32, C.c_int32, C.c_int32] + [_P] * 11 + [C.c_int]
        lib.orc_hmvm_seq2_multi_d.argtypes = ([C.c_int32, C.c_int32, C.c_int32] + [_P] * 10 +
                                              [C.c_int64, _P, C.c_int64, C.c_int32])
        lib.orc_max_threads.restype = C.c_int
        _orc = lib
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_SO)
        for fn in ("ref_load1", "ref_load2"):
            getattr(lib, fn).restype = C.c_void_p
            getattr(lib, fn).argtypes = [C.c_char_p]
        lib.ref_wrap2.restype = C.c_void_p
        lib.ref_wrap2.argtypes = [C.c_int] * 4 + [_P] * 9
        lib.ref_info.argtypes = [C.c_void_p, _P]
        lib.ref_export2.argtypes = [C.c_void_p] + [_P] * 9
        lib.ref_make_float.argtypes = [C.c_void_p]
        for fn in ("ref_seq2_d", "ref_seq2_f"):
            getattr(lib, fn).argtypes = [C.c_void_p, _P, _P, C.c_int]
        lib.ref_seq1_d.argtypes = [C.c_void_p, _P, _P, C.c_int]
        for fn in ("ref_omp2_d", "ref_omp2_f"):
            getattr(lib, fn).argtypes = [C.c_void_p, _P, _P, C.c_int]
        lib.ref_free.argtypes = [C.c_void_p]
        lib.ref_max_threads.restype = C.c_int
        _ref = lib
    return _ref


def _leaf_args(hm):
    arrs = [hm.ltmtx, hm.kt, hm.ndl, hm.ndt, hm.nstrtl, hm.nstrtt, hm.a1, hm.a2]
    return [_p(np.ascontiguousarray(a)) for a in arrs], arrs


def oracle_hmvm(hm, x, a2i: int = 0) -> np.ndarray:
    """hmvm_seq_2<T,a2i> restated (oracle/hmvm_oracle.c); T follows hm.rowmat."""
    lib = oracle_lib()
    args, keep = _leaf_args(hm)
    if hm.rowmat.dtype == np.float32:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(hm.nd, np.float32)
        lib.orc_hmvm_seq2_f(hm.nd, hm.nlf, hm.ktmax, *args, _p(hm.rowmat), _p(x), _p(y), a2i)
    else:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(hm.nd, np.float64)
        lib.orc_hmvm_seq2_d(hm.nd, hm.nlf, hm.ktmax, *args, _p(hm.rowmat), _p(x), _p(y), a2i)
    return y


def oracle_omp(hm, x, nthreads: int = 0) -> np.ndarray:
    lib = oracle_lib()
    args, keep = _leaf_args(hm)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(hm.nd, np.float64)
    lib.orc_omp2_d(hm.nd, hm.nlf, hm.ktmax, *args, _p(hm.rowmat), _p(x), _p(y), nthreads)
    return y


class RefMatrix:
    """The reference's own matrix2<double> (and its float copy) wrapped over an HMatrix."""

    def __init__(self, hm):
        assert hm.rowmat.dtype == np.float64 and hm.fits_matrix2()
        self.lib = ref_lib()
        self._keep = [np.ascontiguousarray(getattr(hm, n), dtype=np.int32)
                      for n in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2")]
        self._rm = hm.rowmat
        self.nd = hm.nd
        self.h = self.lib.ref_wrap2(hm.nd, hm.nlf, hm.ktmax, hm.len, *[_p(a) for a in self._keep], _p(self._rm))
        self._float = False

    def seq2(self, x, a2i=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.nd)
        self.lib.ref_seq2_d(self.h, _p(x), _p(y), a2i)
        return y

    def seq2_f(self, x, a2i=0):
        if not self._float:
            self.lib.ref_make_float(self.h)
            self._float = True
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(self.nd, np.float32)
        self.lib.ref_seq2_f(self.h, _p(x), _p(y), a2i)
        return y

    def omp2(self, x, nthreads=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.nd)
        self.lib.ref_omp2_d(self.h, _p(x), _p(y), nthreads)
        return y

    def close(self):
        if self.h:
            self.lib.ref_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def relerr(y, yref) -> float:
    y = np.asarray(y, dtype=np.float64)
    yref = np.asarray(yref, dtype=np.float64)
    d = np.linalg.norm(yref)
    return float(np.linalg.norm(y - yref) / (d if d > 0 else 1.0))


# ---- CPU emulation of the repacked layout ---------------------------------
def emulate_layout(view, x: np.ndarray) -> np.ndarray:
    """Evaluate y = H x exactly as the tile kernels walk the layout (stage 1
    panels -> t / partial sums, the chunk reduction, stage 2 row tiles)."""
    from hacapk_hmvm_b200 import _lib

    if view.precision == 2:
        return emulate_mixed(view, x)
    VEC = view.vec
    dt = np.float64 if view.precision == 0 else np.float32
    ntiles = view.n_tiles
    tiles = np.ctypeslib.as_array((_lib.TileDesc * ntiles).from_address(view.tiles)) if ntiles else []
    segs = (np.ctypeslib.as_array((_lib.SegDesc * view.n_segs).from_address(view.segs))
            if view.n_segs else [])
    data = np.ctypeslib.as_array((C.c_uint8 * (16 * view.data_vectors)).from_address(view.data)).view(dt) \
        if view.data_vectors else np.zeros(0, dt)
    n_out = max([int(tiles[k]["out_base"]) + int(tiles[k]["nrows"]) for k in range(view.stage1_tiles)
                 if tiles[k]["mode"] == 1] or [0])
    out_idx = np.ctypeslib.as_array(view.out_idx, (n_out,)) if n_out else np.zeros(0, np.int32)
    x = np.asarray(x, dtype=dt)
    t = np.zeros(view.t_len + 16, dt)
    p = np.zeros(view.p_len + 16, dt)
    y = np.full(view.nd, np.nan, dt)

    def run_tile(td):
        R, nvec = int(td["nrows"]), int(td["nvec"])
        off = int(td["data_off"]) * VEC
        M = data[off:off + nvec * R * VEC].reshape(nvec, R, VEC).transpose(1, 0, 2).reshape(R, nvec * VEC)
        z = np.zeros(nvec * VEC, dt)
        col = 0
        for s in range(int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])):
            src, ncols = int(segs[s]["src"]), int(segs[s]["ncols"])
            if src < 0:
                slot = src & 0x7FFFFFFF
                z[col:col + ncols] = t[slot:slot + ncols]
            else:
                z[col:col + ncols] = x[src:src + ncols]
            col += -(-ncols // VEC) * VEC
        return (M.astype(np.float64) @ z.astype(np.float64)).astype(dt)

    for k in range(view.stage1_tiles):
        td = tiles[k]
        acc = run_tile(td)
        R, ob = int(td["nrows"]), int(td["out_base"])
        if td["mode"] == 1:
            t[out_idx[ob:ob + R]] = acc
        else:
            p[ob:ob + R] = acc
    if view.n_red1:
        red = np.ctypeslib.as_array(view.red1, (view.n_red1 * 4,)).reshape(-1, 4)
        for slot, pb, nch, stride in red:
            t[slot] = sum(p[pb + c * stride] for c in range(nch))
    for k in range(view.stage1_tiles, view.n_tiles):
        td = tiles[k]
        acc = run_tile(td)
        R, ob = int(td["nrows"]), int(td["out_base"])
        if td["mode"] == 0:
            y[ob:ob + R] = acc
        else:
            p[ob:ob + R] = acc
    if view.n_red2:
        red = np.ctypeslib.as_array(view.red2, (view.n_red2 * 4,)).reshape(-1, 4)
        for row, pb, nch, stride in red:
            y[row] = sum(p[pb + c * stride] for c in range(nch))
    return y


def _e4m3_table():
    """Values of the 256 OCP FP8 E4M3 (fn) codes."""
    out = np.empty(256)
    for b in range(256):
        e, m = (b >> 3) & 15, b & 7
        s = -1.0 if b & 0x80 else 1.0
        if e == 15 and m == 7:
            out[b] = np.nan
        elif e == 0:
            out[b] = s * m * 2.0 ** -9
        else:
            out[b] = s * (8 + m) * 2.0 ** (e - 10)
    return out


E4M3 = _e4m3_table()


def decode_vectors(raw, ty):
    """raw: uint8 [nv, R, 16] -> float64 [R, nv * elements per vector]."""
    nv, R = raw.shape[:2]
    flat = np.ascontiguousarray(raw).reshape(-1)
    if ty == 0:
        v = flat.view("<f8")
    elif ty == 1:
        v = flat.view("<f4")
    elif ty == 2:
        v = flat.view("<f2")
    elif ty == 4:
        v = (flat.view("<u2").astype(np.uint32) << 16).view("<f4")
    else:
        v = E4M3[flat]
    vs = 16 * v.size // max(flat.size, 1) if flat.size else 1
    return v.astype(np.float64).reshape(nv, R, vs).transpose(1, 0, 2).reshape(R, nv * vs)


def emulate_mixed(view, x: np.ndarray) -> np.ndarray:
    """y = H x for a mixed-precision layout: decodes each segment's stored
    elements, uses x (FP64 segments) or x rounded to FP32 / the FP32 t (other
    segments), scales the V-stage rows and rounds t to FP32 as the kernels do;
    the products are summed in FP64 here (the kernels use FP32 per segment)."""
    from hacapk_hmvm_b200 import _lib
    from layout_checks import SEG_VEC

    tiles = np.ctypeslib.as_array((_lib.TileDesc * view.n_tiles).from_address(view.tiles)) if view.n_tiles else []
    segs = np.ctypeslib.as_array((_lib.SegDesc * view.n_segs).from_address(view.segs)) if view.n_segs else []
    raw = (np.ctypeslib.as_array((C.c_uint8 * (16 * view.data_vectors)).from_address(view.data)).reshape(-1, 16)
           if view.data_vectors else np.zeros((0, 16), np.uint8))
    scale = np.ctypeslib.as_array(view.rowscale, (view.n_rowscale,)) if view.n_rowscale else np.zeros(0)
    n_out = max([int(tiles[k]["out_base"]) + int(tiles[k]["nrows"]) for k in range(view.stage1_tiles)
                 if tiles[k]["mode"] == 1] or [0])
    out_idx = np.ctypeslib.as_array(view.out_idx, (n_out,)) if n_out else np.zeros(0, np.int32)
    x = np.asarray(x, dtype=np.float64)
    x32 = x.astype(np.float32).astype(np.float64)
    t = np.zeros(view.t_len + 16, np.float32)
    p = np.zeros(view.p_len + 16)
    y = np.full(view.nd, np.nan)

    def run_tile(td):
        R = int(td["nrows"])
        v0 = int(td["data_off"])
        row = np.zeros(R)
        for s in range(int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])):
            src, enc = int(segs[s]["src"]), int(segs[s]["ncols"])
            ty, nc = enc >> 28, enc & 0x0FFFFFFF
            nv = -(-nc // SEG_VEC[ty])
            M = decode_vectors(raw[v0:v0 + nv * R].reshape(nv, R, 16), ty)[:, :nc]
            v0 += nv * R
            if src < 0:
                z = t[(src & 0x7FFFFFFF):(src & 0x7FFFFFFF) + nc].astype(np.float64)
            else:
                z = (x if ty == 0 else x32)[src:src + nc]
            row += M @ z
        return row

    for k in range(view.stage1_tiles):
        td = tiles[k]
        R, ob, sb = int(td["nrows"]), int(td["out_base"]), int(td["_pad"])
        val = run_tile(td) * scale[sb:sb + R]
        if td["mode"] == 1:
            t[out_idx[ob:ob + R]] = val.astype(np.float32)
        else:
            p[ob:ob + R] = val
    if view.n_red1:
        red = np.ctypeslib.as_array(view.red1, (view.n_red1 * 4,)).reshape(-1, 4)
        for slot, pb, nch, stride in red:
            t[slot] = np.float32(sum(p[pb + c * stride] for c in range(nch)))
    for k in range(view.stage1_tiles, view.n_tiles):
        td = tiles[k]
        R, ob = int(td["nrows"]), int(td["out_base"])
        acc = run_tile(td)
        if td["mode"] == 0:
            y[ob:ob + R] = acc
        else:
            p[ob:ob + R] = acc
    if view.n_red2:
        red = np.ctypeslib.as_array(view.red2, (view.n_red2 * 4,)).reshape(-1, 4)
        for row, pb, nch, stride in red:
            y[row] = sum(p[pb + c * stride] for c in range(nch))
    return y


def _round16(v, bf16: bool):
    """float32 array -> the nearest FP16 (or BF16) values, ties to even, as float64."""
    v = np.asarray(v, dtype=np.float32)
    if not bf16:
        return v.astype(np.float16).astype(np.float64)
    b = v.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _split16(v, bf16: bool):
    """(hi, lo) of float32 values as the kernels split them: hi = fmt(v),
    lo = fmt(v - hi) with the difference in float32."""
    v = np.asarray(v, dtype=np.float32)
    hi = _round16(v, bf16)
    lo = _round16((v - hi.astype(np.float32)).astype(np.float32), bf16)
    return hi, lo


def emulate_tcw(view, X: np.ndarray) -> np.ndarray:
    """Y = H X (X: [nrhs, N], nrhs <= 128) for a wide tensor-core layout,
    walking its stream as hmvm_tcw_kernel does: per item, per input group
    (consecutive segments with one input range), per K step of 16 columns, per
    segment, per row block in the segment's mask, the block's hi vectors and
    (pair segments) lo vectors; the inputs as scaled 16-bit hi/lo planes; per
    K step hi*x_hi + hi*x_lo (+ lo*x_hi); the V-stage output scaled by 2^-c and
    split into planes, the row stage scaled by s_i and sigma_x.  Products are
    summed in FP64 here (FP32 on the GPU)."""
    from hacapk_hmvm_b200 import _lib

    bf = bool(view.tcw_bf16)
    tiles = np.ctypeslib.as_array((_lib.TileDesc * view.n_tiles).from_address(view.tiles)) if view.n_tiles else []
    segs = np.ctypeslib.as_array((_lib.SegDesc * view.n_segs).from_address(view.segs)) if view.n_segs else []
    blocks = np.ctypeslib.as_array(view.tblocks, (view.n_tiles,)) if view.n_tiles else []
    raw = (np.ctypeslib.as_array((C.c_uint8 * (16 * view.data_vectors)).from_address(view.data))
           if view.data_vectors else np.zeros(0, np.uint8))
    vals = raw.view("<f2").astype(np.float64) if not bf else \
        (raw.view("<u2").astype(np.uint32) << 16).view("<f4").astype(np.float64)
    vals = vals.reshape(-1, 8)  # one 16-byte record per row
    tscale = np.ctypeslib.as_array(view.tscale, (view.n_tscale,)).astype(np.float64) if view.n_tscale else np.zeros(0)
    n1 = view.tscale_rows0
    out_idx = np.ctypeslib.as_array(view.out_idx, (n1,)) if n1 else np.zeros(0, np.int32)
    X = np.asarray(X, dtype=np.float64)
    nr, nd = X.shape
    if bf:
        sig = np.ones(nr)
    else:
        am = np.abs(X.astype(np.float32)).max(axis=1).astype(np.float64)
        sig = np.array([2.0 ** (int(np.ceil(np.log2(m))) - 15) if m > 0 else 1.0 for m in am])
    xi = (X.astype(np.float32) / sig[:, None].astype(np.float32)).astype(np.float32)
    xh, xl = _split16(xi.T, bf)  # [nd, nr]
    th = np.zeros((view.t_len + 1, nr))
    tl = np.zeros((view.t_len + 1, nr))
    part = np.zeros((view.p_len + 1, nr))
    Y = np.full((nr, nd), np.nan)

    def run_item(k):
        td = tiles[k]
        R = [(int(blocks[k]) >> (8 * b)) & 0xFF for b in range(4)]
        brow = np.cumsum([0] + R[:3])
        acc = np.zeros((int(td["nrows"]), nr))
        rec = int(td["data_off"])
        s0, s1 = int(td["seg_begin"]), int(td["seg_begin"]) + int(td["nseg"])
        s = s0
        while s < s1:
            g1 = s + 1
            while g1 < s1 and segs[g1]["src"] == segs[s]["src"] and \
                    (int(segs[g1]["ncols"]) & 0xFFFFFF) == (int(segs[s]["ncols"]) & 0xFFFFFF):
                g1 += 1
            src, nc = int(segs[s]["src"]), int(segs[s]["ncols"]) & 0xFFFFFF
            if src < 0:
                r0 = src & 0x7FFFFFFF
                ah, al = th[r0:r0 + nc], tl[r0:r0 + nc]
            else:
                ah, al = xh[src:src + nc], xl[src:src + nc]
            nv = -(-nc // 8)
            for j in range(-(-nv // 2)):
                nvj = min(2, nv - 2 * j)
                c0, c1 = 16 * j, min(nc, 16 * j + 16)
                for z in range(s, g1):
                    enc = int(segs[z]["ncols"])
                    mask, fmt = (enc >> 24) & 0xF, (enc >> 28) & 1
                    for b in range(4):
                        if not mask >> b & 1:
                            continue
                        Rb = R[b]
                        h = vals[rec:rec + nvj * Rb].reshape(nvj, Rb, 8).transpose(1, 0, 2).reshape(Rb, 8 * nvj)
                        rec += nvj * Rb
                        bh = h[:, :c1 - c0]
                        blk = acc[brow[b]:brow[b] + Rb]
                        blk += bh @ ah[c0:c1] + bh @ al[c0:c1]
                        if fmt:
                            lo = vals[rec:rec + nvj * Rb].reshape(nvj, Rb, 8).transpose(1, 0, 2).reshape(Rb, 8 * nvj)
                            rec += nvj * Rb
                            blk += lo[:, :c1 - c0] @ ah[c0:c1]
            s = g1
        assert rec == int(td["data_off"]) + int(td["nvec"]), (k, rec)
        return acc

    for k in range(view.stage1_tiles):
        td = tiles[k]
        R, ob, sb = int(td["nrows"]), int(td["out_base"]), int(td["_pad"])
        tv = (run_item(k) * tscale[sb:sb + R, None]).astype(np.float32)
        if int(td["mode"]) & 3 == 1:
            h, l = _split16(tv, bf)
            th[out_idx[ob:ob + R]] = h
            tl[out_idx[ob:ob + R]] = l
        else:
            part[ob:ob + R] = tv
    if view.n_red1:
        red = np.ctypeslib.as_array(view.red1, (view.n_red1 * 4,)).reshape(-1, 4)
        for slot, pb, nch, stride in red:
            sm = sum(part[pb + c * stride] for c in range(nch)).astype(np.float32)
            th[slot], tl[slot] = _split16(sm, bf)
    for k in range(view.stage1_tiles, view.n_tiles):
        td = tiles[k]
        R, ob, sb = int(td["nrows"]), int(td["out_base"]), int(td["_pad"])
        acc = run_item(k)
        Y[:, ob:ob + R] = (acc * tscale[sb:sb + R, None] * sig[None, :]).T
    return Y


def layout_for(hm, **opts):
    """Build the host layout of a plan without a GPU; returns (handle, view)."""
    from hacapk_hmvm_b200 import _lib
    from hacapk_hmvm_b200.hmvm import default_opts

    lib = _lib.hmvm_lib()
    opts = dict(opts)
    num_sms = int(opts.pop("num_sms", 148))  # the SM count the plan is laid out for
    o = default_opts(**opts)
    h = C.c_void_p()
    lv = hm.as_leaves64()
    rc = lib.hmvm_b200_layout_build64(C.byref(lv), 1 if hm.rowmat.dtype == np.float32 else 0, C.byref(o),
                                      num_sms, C.byref(h))
    _lib.check(rc, "layout build")
    v = _lib.LayoutView()
    _lib.check(lib.hmvm_b200_layout_view(h, C.byref(v)), "layout view")
    return h, v
