"""HMVM on the GPU through the C ABI (include/hmvm_b200.h).

``Plan``       one H-matrix repacked and resident on the device; ``apply`` runs
               y = H x on device buffers, ``apply_host`` on numpy arrays.
``hmvm``       one-shot y = H x from host arrays (the C ``hmvm_cuda_d/f``).
``hmvm_cuda``  mirror of the reference harness entry point
               ``hmvm_cuda<T>(mat2, b, kernel, dump_result, nbench)``
               (src_hmvm/src_cpp/hmvm_cuda.h:4-7): optional result dump at
               %.3E and a TIME line over nbench timed runs after 5 warm-ups.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .hmatrix import HMatrix

PRECISIONS = {"fp64": _lib.HMVM_FP64, "fp32": _lib.HMVM_FP32, "double": _lib.HMVM_FP64, "float": _lib.HMVM_FP32,
              "mixed": _lib.HMVM_MIXED}
LR_FORMATS = {"fp16": _lib.HMVM_LR_FP16, "bf16": _lib.HMVM_LR_BF16}


def _dev_ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


def _stream_handle(stream):
    if stream is None:
        try:
            import torch

            if torch.cuda.is_available():
                return int(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


def default_opts(**kw) -> _lib.PlanOpts:
    o = _lib.PlanOpts()
    _lib.hmvm_lib().hmvm_b200_default_opts(C.byref(o))
    for k, v in kw.items():
        if v is None:
            continue
        if k == "mixed_lr_format" and isinstance(v, str):
            v = LR_FORMATS[v]
        setattr(o, k, float(v) if isinstance(getattr(o, k), float) else int(v))
    return o


class Plan:
    """A resident, repacked H-matrix on one GPU."""

    def __init__(self, hm: HMatrix, precision: str = "fp64", device: int = -1, **opts):
        lib = _lib.hmvm_lib()
        prec = PRECISIONS[precision]
        o = default_opts(precision=prec, device=device, **opts)
        h = C.c_void_p()
        t0 = time.perf_counter()
        if hm.fits_matrix2():
            m2 = hm.as_matrix2()
            if hm.rowmat.dtype == np.float32:
                rc = lib.hmvm_b200_plan_create_f(C.byref(m2), C.byref(o), C.byref(h))
            else:
                rc = lib.hmvm_b200_plan_create_d(C.byref(m2), C.byref(o), C.byref(h))
        else:
            lv = hm.as_leaves64()
            fn = lib.hmvm_b200_plan_create64_f if hm.rowmat.dtype == np.float32 else lib.hmvm_b200_plan_create64_d
            rc = fn(C.byref(lv), C.byref(o), C.byref(h))
        _lib.check(rc, "plan create")
        self.setup_seconds = time.perf_counter() - t0
        self._h = h
        self.hm = hm
        self.precision = {_lib.HMVM_FP64: "fp64", _lib.HMVM_FP32: "fp32", _lib.HMVM_MIXED: "mixed"}[prec]
        # x and y: FP64 for FP64 and mixed plans, FP32 for FP32 plans
        self.dtype = np.float32 if prec == _lib.HMVM_FP32 else np.float64
        self.nd = hm.nd

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("plan is closed")
        return self._h

    def info(self) -> dict:
        inf = _lib.PlanInfo()
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_get_info(self.handle, C.byref(inf)), "plan info")
        return {f: getattr(inf, f) for f, _ in _lib.PlanInfo._fields_ if not f.startswith("_")}

    def profile(self, enable: bool = True) -> None:
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_profile(self.handle, int(enable)), "profile")

    def profile_read(self) -> tuple[list[float], int]:
        """(summed ms of [V stage, its reduction, row stage, its reduction],
        number of applies)."""
        ms = (C.c_double * 4)()
        n = C.c_int32()
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_profile_read(self.handle, ms, C.byref(n)), "profile_read")
        return [ms[0], ms[1], ms[2], ms[3]], int(n.value)

    def status(self) -> None:
        """Raise if a kernel of this plan reported a device-side error."""
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_status(self.handle), "device status")

    def kernel_count(self) -> int:
        return int(_lib.hmvm_lib().hmvm_b200_plan_kernel_count(self.handle))

    def apply(self, x, y, stream=None) -> None:
        """y = H x; x and y are CUDA tensors (or raw device addresses)."""
        rc = _lib.hmvm_lib().hmvm_b200_apply(self.handle, _dev_ptr(x), _dev_ptr(y), _stream_handle(stream))
        _lib.check(rc, "apply")

    def apply_noalloc(self, x, y, stream=None) -> None:
        """y = H x without any GPU allocation: the scratch comes from the
        library's fixed 16 MiB device array (hmvm_b200_apply_noalloc), for
        callers that may not call cudaMalloc while they run."""
        rc = _lib.hmvm_lib().hmvm_b200_apply_noalloc(self.handle, _dev_ptr(x), _dev_ptr(y), _stream_handle(stream))
        _lib.check(rc, "apply_noalloc")

    def apply_host(self, x: np.ndarray, y: np.ndarray | None = None, stream=None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=self.dtype)
        if x.shape != (self.nd,):
            raise ValueError(f"x must have shape ({self.nd},)")
        if y is None:
            y = np.empty(self.nd, dtype=self.dtype)
        rc = _lib.hmvm_lib().hmvm_b200_apply_host(self.handle, x.ctypes.data, y.ctypes.data,
                                                  _stream_handle(stream) if stream is not None else 0)
        _lib.check(rc, "apply_host")
        return y

    def apply_multi(self, X, Y, stream=None) -> None:
        """Y = H X for a block of right-hand sides: X and Y are CUDA tensors
        of shape (nrhs, N) whose rows are the vectors (column-major N x nrhs
        with leading dimension X.stride(0))."""
        if X.dim() != 2 or Y.shape != X.shape or X.shape[1] != self.nd or X.stride(1) != 1 or Y.stride(1) != 1:
            raise ValueError(f"X and Y must be (nrhs, {self.nd}) with unit stride along N")
        rc = _lib.hmvm_lib().hmvm_b200_apply_multi(self.handle, _dev_ptr(X), X.stride(0), _dev_ptr(Y), Y.stride(0),
                                                   X.shape[0], _stream_handle(stream))
        _lib.check(rc, "apply_multi")

    def apply_multi_host(self, X: np.ndarray, Y: np.ndarray | None = None, stream=None) -> np.ndarray:
        """The same with host arrays of shape (nrhs, N)."""
        X = np.ascontiguousarray(X, dtype=self.dtype)
        if X.ndim != 2 or X.shape[1] != self.nd:
            raise ValueError(f"X must have shape (nrhs, {self.nd})")
        if Y is None:
            Y = np.empty_like(X)
        rc = _lib.hmvm_lib().hmvm_b200_apply_multi_host(self.handle, X.ctypes.data, self.nd, Y.ctypes.data, self.nd,
                                                        X.shape[0],
                                                        _stream_handle(stream) if stream is not None else 0)
        _lib.check(rc, "apply_multi_host")
        return Y

    def capture(self, x, y) -> None:
        """Record y = H x for these CUDA tensors into the plan's CUDA graph
        (hmvm_b200_plan_capture); replay() then runs it with one graph launch."""
        if x.shape != (self.nd,) or y.shape != (self.nd,):
            raise ValueError(f"x and y must have shape ({self.nd},)")
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_capture(self.handle, _dev_ptr(x), _dev_ptr(y)), "plan_capture")

    def replay(self, stream=None) -> None:
        _lib.check(_lib.hmvm_lib().hmvm_b200_plan_replay(self.handle, _stream_handle(stream)), "plan_replay")

    def bicgstab(self, b, u, eps: float = 1e-8, max_steps: int = 1000, stream=None) -> tuple[int, float]:
        """Solve H u = b by BiCGSTAB (hmvm_b200_bicgstab): b, u CUDA tensors,
        u holds the initial guess and receives the solution.  Returns (steps,
        final relative residual)."""
        steps = C.c_int32()
        rel = C.c_double()
        rc = _lib.hmvm_lib().hmvm_b200_bicgstab(self.handle, _dev_ptr(b), _dev_ptr(u), max_steps, eps,
                                                C.byref(steps), C.byref(rel), _stream_handle(stream))
        _lib.check(rc, "bicgstab")
        return steps.value, rel.value

    def gcrm(self, b, u, eps: float = 1e-8, max_steps: int = 1000, restart: int = 20,
             stream=None) -> tuple[int, float]:
        """Solve H u = b by GCR(restart) (hmvm_b200_gcrm); as bicgstab."""
        steps = C.c_int32()
        rel = C.c_double()
        rc = _lib.hmvm_lib().hmvm_b200_gcrm(self.handle, _dev_ptr(b), _dev_ptr(u), max_steps, restart, eps,
                                            C.byref(steps), C.byref(rel), _stream_handle(stream))
        _lib.check(rc, "gcrm")
        return steps.value, rel.value

    def multi_kernel_count(self, nrhs: int) -> int:
        return int(_lib.hmvm_lib().hmvm_b200_plan_multi_kernel_count(self.handle, nrhs))

    def close(self) -> None:
        if self._h:
            _lib.hmvm_lib().hmvm_b200_plan_destroy(self._h)
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


def hmvm(hm: HMatrix, x: np.ndarray, mode: int = 0) -> tuple[np.ndarray, dict]:
    """One-shot y = H x (plan, run, release) through hmvm_cuda_d / hmvm_cuda_f."""
    lib = _lib.hmvm_lib()
    st = _lib.Stats()
    m2 = hm.as_matrix2()
    if hm.rowmat.dtype == np.float32:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(hm.nd, np.float32)
        rc = lib.hmvm_cuda_f(C.byref(m2), x.ctypes.data, y.ctypes.data, int(mode), C.byref(st))
    else:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(hm.nd, np.float64)
        rc = lib.hmvm_cuda_d(C.byref(m2), x.ctypes.data, y.ctypes.data, int(mode), C.byref(st))
    _lib.check(rc, "hmvm_cuda")
    return y, {f: getattr(st, f) for f, _ in _lib.Stats._fields_}


def hmvm_cuda(hm: HMatrix, b: np.ndarray, kernel: int = 0, dump_result: int = 0, nbench: int = 5,
              name: str | None = None) -> np.ndarray:
    """Reference-shaped entry: dump y to result_cuda_b200_<name>.txt at %.3E when
    dump_result, and print ``TIME <nbench> hmvm_cuda_<name> min .. max .. avg ..``
    over nbench timed runs after 5 untimed ones (the reference's M=5 warm-ups,
    hmvm_cuda2.cu:234-302).  Times are device times (CUDA events)."""
    tname = "d" if hm.rowmat.dtype == np.float64 else "f"
    name = name or f"b200_k{kernel}_{tname}"
    with Plan(hm, "fp64" if tname == "d" else "fp32") as plan:
        y = plan.apply_host(b)
        if dump_result:
            with open(f"result_cuda_{name}.txt", "w") as f:
                for v in y:
                    f.write("%.3E\n" % v)
        if nbench > 0:
            import torch

            dt = torch.float64 if tname == "d" else torch.float32
            xd = torch.from_numpy(np.ascontiguousarray(b, dtype=plan.dtype)).to("cuda")
            yd = torch.empty(hm.nd, dtype=dt, device="cuda")
            times = []
            for _ in range(5 + nbench):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                plan.apply(xd, yd)
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1) * 1e-3)
            t = np.array(times[5:])
            print(f"TIME {nbench} hmvm_cuda_{name} min {t.min():e} max {t.max():e} avg {t.mean():e}")
    return y


def autotune(hm: HMatrix, precision: str = "fp64", reps: int = 5, device: int = -1, **base) -> tuple[dict, list]:
    """Time candidate kernel configurations of this matrix's plan on the
    current device (hmvm_b200_autotune64) and return (plan options of the
    fastest measured plan, one dict per candidate timed).  Pass the options
    to Plan(hm, precision, **options)."""
    lib = _lib.hmvm_lib()
    o = default_opts(precision=PRECISIONS[precision], device=device, **base)
    best = _lib.PlanOpts()
    rep = _lib.TuneReport()
    lv = hm.as_leaves64()
    _lib.check(lib.hmvm_b200_autotune64(C.byref(lv), 1 if hm.rowmat.dtype == np.float32 else 0, C.byref(o), reps,
                                        C.byref(best), C.byref(rep)), "autotune")
    keys = ("kernel", "stage1_cfg", "stage2_cfg", "max_tile_rows")
    chosen = {k: getattr(best, k) for k in keys}
    if precision == "mixed":
        chosen.pop("kernel")
    entries = [{f: getattr(rep.entries[i], f) for f, _ in _lib.TuneEntry._fields_ if not f.startswith("_")}
               for i in range(rep.n_entries)]
    for i, e in enumerate(entries):
        e["best"] = i == rep.best_entry
    return chosen, entries


def shape_histogram(hm: HMatrix) -> np.ndarray:
    """The fraction of hm's stored elements in each (kind, rows, width) shape
    class (hmvm_b200_shape_histogram64): 128 bins, dense leaves then low-rank."""
    h = np.zeros(_lib.HMVM_SHAPE_BINS, dtype=np.float32)
    lv = hm.as_leaves64()
    _lib.check(_lib.hmvm_lib().hmvm_b200_shape_histogram64(C.byref(lv), h.ctypes.data_as(C.c_void_p)),
               "shape histogram")
    return h


def autotune_cached(hm: HMatrix, precision: str, cache: str, reps: int = 5, max_distance: float = 0.45,
                    device: int = -1, **base) -> tuple[dict, list, bool]:
    """autotune() through a tuning cache file (hmvm_b200_autotune_cached64): a
    choice stored for this device, precision and factor format whose shape-class
    histogram lies within max_distance of hm's is returned without timing
    anything; otherwise the sweep runs and its choice is appended to the file.
    Returns (plan options, entries, whether the choice came from the cache)."""
    lib = _lib.hmvm_lib()
    o = default_opts(precision=PRECISIONS[precision], device=device, **base)
    best = _lib.PlanOpts()
    rep = _lib.TuneReport()
    hit = C.c_int32(0)
    lv = hm.as_leaves64()
    _lib.check(lib.hmvm_b200_autotune_cached64(C.byref(lv), 1 if hm.rowmat.dtype == np.float32 else 0, C.byref(o),
                                               reps, str(cache).encode(), max_distance, C.byref(best),
                                               C.byref(rep), C.byref(hit)), "autotune")
    keys = ("kernel", "stage1_cfg", "stage2_cfg", "max_tile_rows")
    chosen = {k: getattr(best, k) for k in keys}
    if precision == "mixed":
        chosen.pop("kernel")
    entries = [{f: getattr(rep.entries[i], f) for f, _ in _lib.TuneEntry._fields_ if not f.startswith("_")}
               for i in range(rep.n_entries)]
    for i, e in enumerate(entries):
        e["best"] = i == rep.best_entry
    return chosen, entries, bool(hit.value)
