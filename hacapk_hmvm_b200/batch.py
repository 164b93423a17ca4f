"""Batches of independent H-matrices (hmvm_b200_batch_*): instances grouped by
their right-hand-side count into classes, each one block-diagonal plan over its
instances' concatenated index space, so every stage of a class is one
persistent launch over all its instances; apply() runs the classes directly,
capture()/launch() replay them as one CUDA graph."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .hmatrix import HMatrix
from .hmvm import PRECISIONS, _dev_ptr, _stream_handle, default_opts


class Batch:
    def __init__(self, mats: list[HMatrix], precision: str = "fp32", device: int = -1,
                 nrhs: list[int] | None = None, **opts):
        """nrhs: right-hand sides each instance will be applied with (groups the
        instances into pass-width classes); None = opts' nrhs_max for all."""
        lib = _lib.hmvm_lib()
        prec = PRECISIONS[precision]
        o = default_opts(precision=prec, device=device, **opts)
        if not mats:
            raise ValueError("a batch needs at least one matrix")
        f32 = mats[0].rowmat.dtype == np.float32
        if any((m.rowmat.dtype == np.float32) != f32 for m in mats):
            raise TypeError("all matrices of a batch store the same element type")
        self._lv = (_lib.Leaves64 * len(mats))(*[m.as_leaves64() for m in mats])
        h = C.c_void_p()
        fn = lib.hmvm_b200_batch_create64_f if f32 else lib.hmvm_b200_batch_create64_d
        nr = None if nrhs is None else (C.c_int32 * len(mats))(*[int(k) for k in nrhs])
        _lib.check(fn(self._lv, len(mats), C.byref(o), nr, C.byref(h)), "batch create")
        self._h = h
        self.mats = mats
        self.n = [m.nd for m in mats]
        self.precision = precision
        self.dtype = np.float32 if prec == _lib.HMVM_FP32 else np.float64
        self._keep = None

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("batch is closed")
        return self._h

    def info(self) -> dict:
        inf = _lib.PlanInfo()
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_get_info(self.handle, C.byref(inf)), "batch info")
        return {f: getattr(inf, f) for f, _ in _lib.PlanInfo._fields_ if not f.startswith("_")}

    def _tables(self, Xs, Ys):
        """Xs, Ys: per instance CUDA tensors of shape (nrhs_m, N_m) (rows = vectors)."""
        k = len(self.n)
        if len(Xs) != k or len(Ys) != k:
            raise ValueError(f"need {k} X and Y blocks")
        X = (C.c_void_p * k)(*[_dev_ptr(x) for x in Xs])
        Y = (C.c_void_p * k)(*[_dev_ptr(y) for y in Ys])
        ldx = (C.c_int64 * k)(*[x.stride(0) if x.dim() == 2 else self.n[i] for i, x in enumerate(Xs)])
        ldy = (C.c_int64 * k)(*[y.stride(0) if y.dim() == 2 else self.n[i] for i, y in enumerate(Ys)])
        nr = (C.c_int32 * k)(*[(x.shape[0] if x.dim() == 2 else 1) for x in Xs])
        for i, (x, y) in enumerate(zip(Xs, Ys)):
            if x.shape != y.shape or x.shape[-1] != self.n[i] or x.stride(-1) != 1 or y.stride(-1) != 1:
                raise ValueError(f"instance {i}: X and Y must be (nrhs, {self.n[i]}) with unit stride along N")
        return X, ldx, Y, ldy, nr

    def apply(self, Xs, Ys, stream=None) -> None:
        t = self._tables(Xs, Ys)
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_apply(self.handle, *t, _stream_handle(stream)), "batch apply")

    def capture(self, Xs, Ys) -> None:
        t = self._tables(Xs, Ys)
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_capture(self.handle, *t), "batch capture")
        self._keep = (Xs, Ys)  # the graph holds their addresses

    def launch(self, stream=None) -> None:
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_launch(self.handle, _stream_handle(stream)), "batch launch")

    def status(self) -> None:
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_status(self.handle), "batch status")

    def kernel_count(self) -> int:
        """Kernels one apply / graph replay launches for the columns last given."""
        return int(_lib.hmvm_lib().hmvm_b200_batch_kernel_count(self.handle))

    def class_count(self) -> int:
        return int(_lib.hmvm_lib().hmvm_b200_batch_class_count(self.handle))

    def instance(self, m: int) -> tuple[int, int, int]:
        """(N, class, row offset within the class's plan) of instance m."""
        n, c, off = C.c_int32(), C.c_int32(), C.c_int64()
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_instance(self.handle, m, C.byref(n), C.byref(c), C.byref(off)),
                   "batch instance")
        return n.value, c.value, off.value

    def close(self) -> None:
        if self._h:
            _lib.hmvm_lib().hmvm_b200_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
