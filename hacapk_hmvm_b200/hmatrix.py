"""H-matrix leaf tables on the host.

``HMatrix`` holds the SoA leaf table of the reference's ``matrix2<T>``
(src_hmvm/src_cpp/hacapk.h:23-36) as numpy arrays with 64-bit offsets, and
converts it to the C structures the library takes.  Matrices come from

* ``HMatrix.load(path)``      hmatrix_1.bin / hmatrix_2.bin through the
                              library's loaders (replacing loadHmatrix /
                              loadHmatrix2, src_hmvm/src_cpp/loadmatrix.cpp),
                              and the 64-bit variant of hmatrix_2.bin;
* ``HMatrix.generate(...)``   the HACApK-rule generator (include/hacapk_hgen.h).
"""
from __future__ import annotations

import ctypes as C
import functools
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _lib

GEOMETRIES = {"sphere": 0, "cube": 1, "cube_surface": 1, "plate": 2, "plate_2x1": 2}


def _np_from_owned(ptr, n, dtype, owner=None):
    """An array over n elements of C memory at ptr.  With `owner` (the object
    whose lifetime frees that memory), the array and every view of it keep the
    owner alive."""
    if n == 0:
        return np.zeros(0, dtype)
    buf = (C.c_ubyte * (n * np.dtype(dtype).itemsize)).from_address(C.cast(ptr, C.c_void_p).value)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dtype)


_np_from = _np_from_owned


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class HMatrix:
    nd: int
    ktmax: int
    ltmtx: np.ndarray
    kt: np.ndarray
    ndl: np.ndarray
    ndt: np.ndarray
    nstrtl: np.ndarray
    nstrtt: np.ndarray
    a1: np.ndarray  # int64 element offsets
    a2: np.ndarray
    rowmat: np.ndarray  # float64 or float32
    meta: dict = field(default_factory=dict)
    _keep: list = field(default_factory=list, repr=False)

    # ---- basic properties ------------------------------------------------
    @property
    def nlf(self) -> int:
        return int(self.ltmtx.shape[0])

    @property
    def len(self) -> int:
        return int(self.rowmat.shape[0])

    @property
    def dtype(self):
        return self.rowmat.dtype

    def stored_elements(self) -> int:
        lr = self.ltmtx == 1
        return int((self.kt[lr].astype(np.int64) * (self.ndl[lr] + self.ndt[lr])).sum()
                   + (self.ndl[~lr].astype(np.int64) * self.ndt[~lr]).sum())

    def algorithmic_bytes(self, elem_bytes: int | None = None, nrhs: int = 1) -> int:
        """Stored leaf elements once plus each x and y element once."""
        e = elem_bytes if elem_bytes is not None else self.rowmat.itemsize
        return self.stored_elements() * e + 2 * nrhs * self.nd * e

    # ---- constructors ----------------------------------------------------
    @classmethod
    def from_arrays(cls, nd, ktmax, ltmtx, kt, ndl, ndt, nstrtl, nstrtt, a1, a2, rowmat, meta=None) -> "HMatrix":
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        i64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)
        rm = np.ascontiguousarray(rowmat)
        if rm.dtype not in (np.float64, np.float32):
            rm = rm.astype(np.float64)
        return cls(int(nd), int(ktmax), i32(ltmtx), i32(kt), i32(ndl), i32(ndt), i32(nstrtl), i32(nstrtt),
                   i64(a1), i64(a2), rm, dict(meta or {}))

    @classmethod
    def generate(cls, n: int, geometry: str | int = "sphere", leaf_size: int = 32, eta: float = 2.0,
                 eps: float = 1e-4, seed: int = 1, kmax: int = 1000, aca_eps_factor: float = 1e-3,
                 nthreads: int = 0, fill: str = "cpu", device: int = 0) -> "HMatrix":
        """An H-matrix of the point kernel built with HACApK's rules.  `fill`:
        "cpu" fills the leaves on the host (hgen_fill_leaves, OpenMP); "gpu" on
        `device` (hmvm_b200_aca_fill; bit-identical leaf data, report in
        meta["aca_report"])."""
        if fill not in ("cpu", "gpu"):
            raise ValueError("fill must be 'cpu' or 'gpu'")
        lib = _lib.hgen_lib()
        p = _lib.HgenParams()
        lib.hgen_default_params(C.byref(p))
        p.n = int(n)
        p.geometry = GEOMETRIES[geometry] if isinstance(geometry, str) else int(geometry)
        p.leaf_size = int(leaf_size)
        p.eta = float(eta)
        p.eps = float(eps)
        p.seed = int(seed)
        p.kmax = int(kmax)
        p.aca_eps_factor = float(aca_eps_factor)
        p.nthreads = int(nthreads)
        mp = C.POINTER(_lib.HgenMatrix)()
        rc = lib.hgen_build_tree(C.byref(p), C.byref(mp))
        if rc != 0:
            raise RuntimeError(f"hgen_build_tree failed with status {rc}")
        report = None
        if fill == "cpu":
            rc = lib.hgen_fill_leaves(mp, C.byref(p))
            where = "hgen_fill_leaves"
        else:
            report = _lib.AcaReport()
            rc = _lib.hmvm_lib().hmvm_b200_aca_fill(mp, C.byref(p), int(device), C.byref(report))
            where = "hmvm_b200_aca_fill"
        if rc != 0:
            lib.hgen_free(mp)
            if fill == "gpu":
                _lib.check(rc, where)
            raise RuntimeError(f"{where} failed with status {rc}")
        obj = cls._wrap_hgen(mp, dict(n=int(n), geometry=geometry, leaf_size=leaf_size, eta=eta, eps=eps,
                                      seed=seed, kmax=kmax, aca_eps_factor=aca_eps_factor))
        if report is not None:
            obj.meta["aca_report"] = {f: getattr(report, f) for f, _ in _lib.AcaReport._fields_}
        return obj

    @classmethod
    def from_mesh(cls, path: str, eps: float = 1e-6, leaf_size: int = 15, eta: float = 2.0, kmax: int = 1000,
                  aca_eps_factor: float = 1e-3, nthreads: int = 0) -> "HMatrix":
        """The ppohBEM collocation H-matrix of a .pbf triangle mesh
        (hgen_read_pbf + hgen_build_tree_mesh + hgen_fill_leaves); the defaults
        are HACApK's with the reference driver's tolerance 1e-6."""
        lib = _lib.hgen_lib()
        mesh = C.POINTER(_lib.HgenMesh)()
        rc = lib.hgen_read_pbf(path.encode(), C.byref(mesh))
        if rc != 0:
            raise OSError(f"hgen_read_pbf({path}) failed with status {rc}")
        mesh_owner = _COwner(mesh, lib.hgen_free_mesh)
        p = _lib.HgenParams()
        lib.hgen_default_params(C.byref(p))
        p.leaf_size, p.eta, p.eps, p.kmax = int(leaf_size), float(eta), float(eps), int(kmax)
        p.aca_eps_factor, p.nthreads = float(aca_eps_factor), int(nthreads)
        mp = C.POINTER(_lib.HgenMatrix)()
        rc = lib.hgen_build_tree_mesh(C.byref(p), mesh, C.byref(mp))
        if rc != 0:
            raise RuntimeError(f"hgen_build_tree_mesh failed with status {rc}")
        rc = lib.hgen_fill_leaves(mp, C.byref(p))
        if rc != 0:
            lib.hgen_free(mp)
            raise RuntimeError(f"hgen_fill_leaves failed with status {rc}")
        obj = cls._wrap_hgen(mp, dict(mesh=path, leaf_size=leaf_size, eta=eta, eps=eps, kmax=kmax,
                                      aca_eps_factor=aca_eps_factor))
        obj._keep.append(mesh_owner)  # entry() evaluates the mesh kernel
        return obj

    @classmethod
    def _wrap_hgen(cls, mp, gen_meta) -> "HMatrix":
        """An HMatrix over a filled hgen_hmatrix (arrays owned by it)."""
        lib = _lib.hgen_lib()
        m = mp.contents
        nlf = m.nlf
        owner = _COwner(mp, lib.hgen_free)
        _np_from = functools.partial(_np_from_owned, owner=owner)
        obj = cls(
            nd=m.nd, ktmax=m.ktmax,
            ltmtx=_np_from(m.ltmtx, nlf, np.int32), kt=_np_from(m.kt, nlf, np.int32),
            ndl=_np_from(m.ndl, nlf, np.int32), ndt=_np_from(m.ndt, nlf, np.int32),
            nstrtl=_np_from(m.nstrtl, nlf, np.int32), nstrtt=_np_from(m.nstrtt, nlf, np.int32),
            a1=_np_from(m.a1, nlf, np.int64), a2=_np_from(m.a2, nlf, np.int64),
            rowmat=_np_from(m.rowmat, m.len, np.float64),
            meta=dict(generator=gen_meta, n_lowrank=int(m.n_lowrank), n_dense=int(m.n_dense),
                      aca_incomplete=int(m.aca_incomplete)),
        )
        obj.meta["lod"] = _np_from(m.lod, m.nd, np.int32)
        obj.meta["coords"] = _np_from(m.coords, 3 * m.nd, np.float64).reshape(-1, 3)
        obj._keep.append(owner)
        obj._hgen_ptr = mp
        return obj

    @classmethod
    def load(cls, path: str, fmt: int | None = None, wide: bool = False) -> "HMatrix":
        """Read hmatrix_1.bin (fmt=1), hmatrix_2.bin (fmt=2) or its 64-bit variant
        (fmt=3); fmt=None guesses from the header record length (12, 16 or 20
        bytes).  Formats 1 and 2 go through the reference-signature loaders
        (int offsets) unless `wide`; format 3, and `wide`, through
        hmvm_b200_load_leaves64 (64-bit offsets, no element-count ceiling)."""
        if fmt is None:
            with open(path, "rb") as f:
                head = np.frombuffer(f.read(4), dtype=np.int32)
            fmt = {16: 2, 20: 3}.get(int(head[0]) if head.size else 12, 1)
        lib = _lib.hmvm_lib()
        if fmt == 3 or wide:
            return cls._load_wide(path)
        m2 = _lib.Matrix2_d()
        if fmt == 1:
            rc = lib.hmvm_b200_load_hmatrix(path.encode(), None, C.byref(m2))
        else:
            rc = lib.hmvm_b200_load_hmatrix2(path.encode(), C.byref(m2))
        _lib.check(rc, f"load {path}")
        try:
            nlf = m2.nlf
            obj = cls.from_arrays(
                m2.nd, m2.ktmax, _np_from(m2.ltmtx, nlf, np.int32).copy(), _np_from(m2.kt, nlf, np.int32).copy(),
                _np_from(m2.ndl, nlf, np.int32).copy(), _np_from(m2.ndt, nlf, np.int32).copy(),
                _np_from(m2.nstrtl, nlf, np.int32).copy(), _np_from(m2.nstrtt, nlf, np.int32).copy(),
                _np_from(m2.a1, nlf, np.int32).astype(np.int64), _np_from(m2.a2, nlf, np.int32).astype(np.int64),
                _np_from(m2.rowmat, m2.len, np.float64).copy(), meta=dict(source=path, format=fmt))
        finally:
            lib.hmvm_b200_free_matrix2_d(C.byref(m2))
        return obj

    @classmethod
    def _load_wide(cls, path: str) -> "HMatrix":
        lib = _lib.hmvm_lib()
        lv = _lib.Leaves64()
        fmt = C.c_int32(0)
        _lib.check(lib.hmvm_b200_load_leaves64(path.encode(), C.byref(lv), C.byref(fmt)), f"load {path}")
        keep = _lib.Leaves64()
        C.memmove(C.byref(keep), C.byref(lv), C.sizeof(lv))
        owner = _COwner(C.pointer(keep), lib.hmvm_b200_free_leaves64)
        nlf = lv.nlf
        arr = functools.partial(_np_from_owned, owner=owner)
        return cls.from_arrays(
            lv.nd, lv.ktmax, arr(lv.ltmtx, nlf, np.int32), arr(lv.kt, nlf, np.int32), arr(lv.ndl, nlf, np.int32),
            arr(lv.ndt, nlf, np.int32), arr(lv.nstrtl, nlf, np.int32), arr(lv.nstrtt, nlf, np.int32),
            arr(lv.a1, nlf, np.int64), arr(lv.a2, nlf, np.int64), arr(lv.rowmat, lv.len, np.float64),
            meta=dict(source=path, format=int(fmt.value)))

    # ---- conversions -----------------------------------------------------
    def to_float(self) -> "HMatrix":
        """FP32 copy (element-wise rounding, as convertD2F)."""
        # copies of the index arrays: they may be views of memory this matrix owns
        return HMatrix.from_arrays(self.nd, self.ktmax, *(a.copy() for a in (
            self.ltmtx, self.kt, self.ndl, self.ndt, self.nstrtl, self.nstrtt, self.a1, self.a2)),
            self.rowmat.astype(np.float32), self.meta)

    def fits_matrix2(self) -> bool:
        return self.len <= np.iinfo(np.int32).max

    def as_matrix2(self):
        """A Matrix2_d / Matrix2_f view of the arrays (int32 offsets; rowmat_t NULL)."""
        if not self.fits_matrix2():
            raise OverflowError("stored elements exceed matrix2's int len; use as_leaves64()")
        a1 = self.a1.astype(np.int32)
        a2 = self.a2.astype(np.int32)
        isf = self.rowmat.dtype == np.float32
        m = (_lib.Matrix2_f if isf else _lib.Matrix2_d)()
        m.nd, m.nlf, m.ktmax, m.len = self.nd, self.nlf, self.ktmax, self.len
        for name in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt"):
            setattr(m, name, _ptr(getattr(self, name), C.c_int))
        m.a1 = _ptr(a1, C.c_int)
        m.a2 = _ptr(a2, C.c_int)
        m.rowmat = _ptr(self.rowmat, C.c_float if isf else C.c_double)
        m._keep = (a1, a2, self)
        return m

    def as_leaves64(self):
        lv = _lib.Leaves64()
        lv.nd, lv.nlf, lv.ktmax, lv.len = self.nd, self.nlf, self.ktmax, self.len
        for name in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt"):
            setattr(lv, name, _ptr(getattr(self, name), C.c_int32))
        lv.a1 = _ptr(self.a1, C.c_int64)
        lv.a2 = _ptr(self.a2, C.c_int64)
        lv.rowmat = self.rowmat.ctypes.data
        lv._keep = self
        return lv

    def _as_hgen(self):
        if self.rowmat.dtype != np.float64:
            raise TypeError("the .bin writers store FP64 elements")
        m = _lib.HgenMatrix()
        m.nd, m.nlf, m.ktmax, m.len = self.nd, self.nlf, self.ktmax, self.len
        for name in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt"):
            setattr(m, name, _ptr(getattr(self, name), C.c_int32))
        m.a1 = _ptr(self.a1, C.c_int64)
        m.a2 = _ptr(self.a2, C.c_int64)
        m.rowmat = _ptr(self.rowmat, C.c_double)
        m._keep = self
        return m

    def write_bin1(self, path: str) -> None:
        rc = _lib.hgen_lib().hgen_write_bin1(C.byref(self._as_hgen()), path.encode())
        if rc != 0:
            raise OSError(f"hgen_write_bin1 failed with status {rc}")

    def write_bin2(self, path: str) -> None:
        rc = _lib.hgen_lib().hgen_write_bin2(C.byref(self._as_hgen()), path.encode())
        if rc != 0:
            raise OSError(f"hgen_write_bin2 failed with status {rc}")

    def write_bin64(self, path: str) -> None:
        """hmatrix_2.bin with a 64-bit len in the header (format 3)."""
        rc = _lib.hgen_lib().hgen_write_bin64(C.byref(self._as_hgen()), path.encode())
        if rc != 0:
            raise OSError(f"hgen_write_bin64 failed with status {rc}")

    def entry(self, ill: int, itt: int) -> float:
        """Exact kernel entry at 1-based permuted positions (generated matrices only)."""
        return _lib.hgen_lib().hgen_entry(self._hgen_ptr, int(ill), int(itt))

    def dense(self) -> np.ndarray:
        """The full nd x nd matrix the leaves represent (small matrices only)."""
        A = np.zeros((self.nd, self.nd), dtype=np.float64)
        rm = self.rowmat.astype(np.float64)
        for i in range(self.nlf):
            r0, c0, ndl, ndt = self.nstrtl[i] - 1, self.nstrtt[i] - 1, self.ndl[i], self.ndt[i]
            if self.ltmtx[i] == 1:
                k = self.kt[i]
                V = rm[self.a1[i]:self.a1[i] + k * ndt].reshape(k, ndt)
                U = rm[self.a2[i]:self.a2[i] + k * ndl].reshape(k, ndl)
                A[r0:r0 + ndl, c0:c0 + ndt] += U.T @ V
            else:
                A[r0:r0 + ndl, c0:c0 + ndt] += rm[self.a1[i]:self.a1[i] + ndl * ndt].reshape(ndl, ndt)
        return A


class _COwner:
    """Frees a C allocation when the last Python reference goes away."""

    def __init__(self, ptr, free_fn):
        self._fin = weakref.finalize(self, free_fn, ptr)
