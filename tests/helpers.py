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
SAMPLE_BIN = "/root/reference/src_hdump/hmatrix_sample.bin"

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


def layout_for(hm, **opts):
    """Build the host layout of a plan without a GPU; returns (handle, view)."""
    from hacapk_hmvm_b200 import _lib
    from hacapk_hmvm_b200.hmvm import default_opts

    lib = _lib.hmvm_lib()
    o = default_opts(**opts)
    h = C.c_void_p()
    lv = hm.as_leaves64()
    rc = lib.hmvm_b200_layout_build64(C.byref(lv), 1 if hm.rowmat.dtype == np.float32 else 0, C.byref(o),
                                      int(opts.get("num_sms", 148)) if "num_sms" in opts else 148, C.byref(h))
    _lib.check(rc, "layout build")
    v = _lib.LayoutView()
    _lib.check(lib.hmvm_b200_layout_view(h, C.byref(v)), "layout view")
    return h, v
