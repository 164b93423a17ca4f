"""ctypes bindings for include/hmvm_b200.h and include/hacapk_hgen.h.

The shared libraries are built in-tree (``hacapk_hmvm_b200/build.py``).  There
is no Python fallback: if a library is missing, loading raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
# HMVM_B200_DEVICE_CHECKS=1 selects the build with device bounds checks
# (hmvm_b200_layout_validate's checks before every single-vector stage launch)
DEVICE_CHECKS = os.environ.get("HMVM_B200_DEVICE_CHECKS", "0") == "1"
LIB_HMVM_PATH = os.path.join(_PKG, "libhmvm_b200_checked.so" if DEVICE_CHECKS else "libhmvm_b200.so")
LIB_HGEN_PATH = os.path.join(_PKG, "libhgen.so")

# ---- status codes (hmvm_b200.h) ------------------------------------------
HMVM_OK = 0
HMVM_EINVAL = -1
HMVM_ENOMEM = -2
HMVM_ECUDA = -3
HMVM_EIO = -4
HMVM_EFORMAT = -5
HMVM_ERANGE = -6
HMVM_ENODEV = -7
HMVM_EDEVICE = -8

HMVM_FP64 = 0
HMVM_FP32 = 1
HMVM_MIXED = 2
HMVM_LR_FP16 = 0
HMVM_LR_BF16 = 1
# storage types of mixed-plan segments (high bits of hmvm_seg_desc.ncols)
ST_F64, ST_F32, ST_F16, ST_E4M3, ST_BF16 = 0, 1, 2, 3, 4
SEG_TYPE_SHIFT = 28

HMVM_NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024

_ip = C.POINTER(C.c_int)


class Submatrix_d(C.Structure):
    _fields_ = [("ltmtx", C.c_int), ("kt", C.c_int), ("ndl", C.c_int), ("ndt", C.c_int),
                ("nstrtl", C.c_int), ("nstrtt", C.c_int),
                ("a1", C.POINTER(C.c_double)), ("a2", C.POINTER(C.c_double)), ("a2t", C.POINTER(C.c_double))]


class Submatrix_f(C.Structure):
    _fields_ = [("ltmtx", C.c_int), ("kt", C.c_int), ("ndl", C.c_int), ("ndt", C.c_int),
                ("nstrtl", C.c_int), ("nstrtt", C.c_int),
                ("a1", C.POINTER(C.c_float)), ("a2", C.POINTER(C.c_float)), ("a2t", C.POINTER(C.c_float))]


class Matrix_d(C.Structure):
    _fields_ = [("nd", C.c_int), ("nlf", C.c_int), ("ktmax", C.c_int), ("nleavs", _ip),
                ("submat", C.POINTER(Submatrix_d)),
                ("b1", C.c_int), ("b2", C.c_int), ("b3", C.c_int), ("e1", C.c_int), ("e2", C.c_int), ("e3", C.c_int)]


class Matrix_f(C.Structure):
    _fields_ = [("nd", C.c_int), ("nlf", C.c_int), ("ktmax", C.c_int), ("nleavs", _ip),
                ("submat", C.POINTER(Submatrix_f)),
                ("b1", C.c_int), ("b2", C.c_int), ("b3", C.c_int), ("e1", C.c_int), ("e2", C.c_int), ("e3", C.c_int)]


def _matrix2_fields(elem):
    return [("nd", C.c_int), ("nlf", C.c_int), ("ktmax", C.c_int), ("len", C.c_int), ("nleavs", _ip),
            ("ltmtx", _ip), ("kt", _ip), ("ndl", _ip), ("ndt", _ip), ("nstrtl", _ip), ("nstrtt", _ip),
            ("a1", _ip), ("a2", _ip), ("rowmat", C.POINTER(elem)), ("rowmat_t", C.POINTER(elem)),
            ("napprox", C.c_int), ("ndense", C.c_int), ("approx", _ip), ("dense", _ip)]


class Matrix2_d(C.Structure):
    _fields_ = _matrix2_fields(C.c_double)


class Matrix2_f(C.Structure):
    _fields_ = _matrix2_fields(C.c_float)


class Leaves64(C.Structure):
    _fields_ = [("nd", C.c_int32), ("nlf", C.c_int32), ("ktmax", C.c_int32), ("_pad0", C.c_int32),
                ("len", C.c_int64),
                ("ltmtx", C.POINTER(C.c_int32)), ("kt", C.POINTER(C.c_int32)), ("ndl", C.POINTER(C.c_int32)),
                ("ndt", C.POINTER(C.c_int32)), ("nstrtl", C.POINTER(C.c_int32)), ("nstrtt", C.POINTER(C.c_int32)),
                ("a1", C.POINTER(C.c_int64)), ("a2", C.POINTER(C.c_int64)), ("rowmat", C.c_void_p)]


class PlanOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("max_tile_rows", C.c_int32),
                ("split_cols", C.c_int32), ("stage1_cfg", C.c_int32), ("stage2_cfg", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("kernel", C.c_int32), ("mixed_fp8_eps", C.c_double),
                ("mixed_fp32_tau", C.c_double), ("mixed_lr_format", C.c_int32), ("nrhs_max", C.c_int32)]


class PlanInfo(C.Structure):
    _fields_ = [("nd", C.c_int32), ("nlf", C.c_int32), ("n_lowrank", C.c_int32), ("n_dense", C.c_int32),
                ("precision", C.c_int32), ("device", C.c_int32), ("num_sms", C.c_int32), ("_pad0", C.c_int32),
                ("algorithmic_bytes", C.c_int64), ("device_bytes", C.c_int64), ("t_len", C.c_int64),
                ("stage1_tiles", C.c_int32), ("stage2_tiles", C.c_int32), ("stage1_teams", C.c_int32),
                ("stage2_teams", C.c_int32), ("split_rows", C.c_int32), ("kernels_per_apply", C.c_int32),
                ("stage1_cfg", C.c_int32), ("stage2_cfg", C.c_int32), ("flops", C.c_int64),
                ("stage1_bytes", C.c_int64), ("stage2_bytes", C.c_int64),
                ("kernel", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("cols_fp32", C.c_int64), ("cols_lr16", C.c_int64), ("cols_fp8", C.c_int64),
                ("stage2_ctas_per_sm", C.c_int32), ("nrhs_max", C.c_int32)]


TUNE_MAX_ENTRIES = 64


HMVM_SHAPE_BINS = 128  # include/hmvm_b200.h


class TuneEntry(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("stage1_cfg", C.c_int32), ("stage2_cfg", C.c_int32),
                ("max_tile_rows", C.c_int32), ("ctas_per_sm", C.c_int32), ("_pad0", C.c_int32),
                ("stage1_ms", C.c_double), ("stage2_ms", C.c_double), ("total_ms", C.c_double)]


class TuneReport(C.Structure):
    _fields_ = [("n_entries", C.c_int32), ("best_entry", C.c_int32), ("entries", TuneEntry * TUNE_MAX_ENTRIES)]


class Stats(C.Structure):
    _fields_ = [("seconds_setup", C.c_double), ("seconds_apply", C.c_double),
                ("algorithmic_bytes", C.c_int64), ("gbytes_per_s", C.c_double)]


class TileDesc(C.Structure):
    _fields_ = [("data_off", C.c_int64), ("seg_begin", C.c_int32), ("nseg", C.c_int32), ("nvec", C.c_int32),
                ("out_base", C.c_int32), ("nrows", C.c_int16), ("mode", C.c_int16), ("_pad", C.c_int32)]


class SegDesc(C.Structure):
    _fields_ = [("src", C.c_int32), ("ncols", C.c_int32)]


class LayoutView(C.Structure):
    _fields_ = [("precision", C.c_int32), ("vec", C.c_int32), ("n_tiles", C.c_int32), ("n_segs", C.c_int32),
                ("stage1_tiles", C.c_int32), ("stage2_tiles", C.c_int32), ("stage1_teams", C.c_int32),
                ("stage2_teams", C.c_int32), ("n_red1", C.c_int32), ("n_red2", C.c_int32), ("nd", C.c_int32),
                ("kernel", C.c_int32),
                ("data_vectors", C.c_int64), ("t_len", C.c_int64), ("p_len", C.c_int64),
                ("tiles", C.c_void_p), ("segs", C.c_void_p), ("team_begin1", C.POINTER(C.c_int32)),
                ("team_begin2", C.POINTER(C.c_int32)), ("out_idx", C.POINTER(C.c_int32)),
                ("red1", C.POINTER(C.c_int32)), ("red2", C.POINTER(C.c_int32)), ("data", C.c_void_p),
                ("rowscale", C.POINTER(C.c_double)), ("n_rowscale", C.c_int64),
                ("tcw", C.c_int32), ("tcw_bf16", C.c_int32), ("tscale", C.POINTER(C.c_float)),
                ("n_tscale", C.c_int64), ("tscale_rows0", C.c_int32), ("_pad_view", C.c_int32),
                ("tblocks", C.POINTER(C.c_int32)), ("tgroups", C.POINTER(C.c_uint32)),
                ("tops", C.POINTER(C.c_uint32)), ("tgfirst", C.POINTER(C.c_int32)), ("n_tgroups", C.c_int64),
                ("n_tops", C.c_int64)]


class HgenParams(C.Structure):
    _fields_ = [("n", C.c_int64), ("geometry", C.c_int32), ("leaf_size", C.c_int32), ("eta", C.c_double),
                ("eps", C.c_double), ("aca_eps_factor", C.c_double), ("kmax", C.c_int32),
                ("nthreads", C.c_int32), ("seed", C.c_uint64)]


class HgenMesh(C.Structure):
    _fields_ = [("nond", C.c_int32), ("nofc", C.c_int32), ("nond_on_face", C.c_int32), ("nint_para_fc", C.c_int32),
                ("ndble_para_fc", C.c_int32), ("_pad0", C.c_int32), ("nodes", C.POINTER(C.c_double)),
                ("face2node", C.POINTER(C.c_int32)), ("int_para_fc", C.POINTER(C.c_int32)),
                ("dble_para_fc", C.POINTER(C.c_double))]


class HgenMatrix(C.Structure):
    _fields_ = [("nd", C.c_int32), ("nlf", C.c_int32), ("ktmax", C.c_int32), ("_pad0", C.c_int32),
                ("len", C.c_int64),
                ("ltmtx", C.POINTER(C.c_int32)), ("kt", C.POINTER(C.c_int32)), ("ndl", C.POINTER(C.c_int32)),
                ("ndt", C.POINTER(C.c_int32)), ("nstrtl", C.POINTER(C.c_int32)), ("nstrtt", C.POINTER(C.c_int32)),
                ("a1", C.POINTER(C.c_int64)), ("a2", C.POINTER(C.c_int64)), ("rowmat", C.POINTER(C.c_double)),
                ("lod", C.POINTER(C.c_int32)), ("coords", C.POINTER(C.c_double)),
                ("n_lowrank", C.c_int64), ("n_dense", C.c_int64), ("aca_incomplete", C.c_int64),
                ("mesh", C.POINTER(HgenMesh))]


class AcaReport(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("ktmax", C.c_int32), ("scratch_bytes", C.c_int64),
                ("ms_aca", C.c_double), ("ms_dense", C.c_double), ("ms_gather_copy", C.c_double)]


# Every C symbol declared in include/hmvm_b200.h, with (restype, argtypes).
HMVM_SIGNATURES = {
    "hmvm_b200_load_hmatrix": (C.c_int, [C.c_char_p, C.POINTER(Matrix_d), C.POINTER(Matrix2_d)]),
    "hmvm_b200_load_hmatrix2": (C.c_int, [C.c_char_p, C.POINTER(Matrix2_d)]),
    "hmvm_b200_load_leaves64": (C.c_int, [C.c_char_p, C.POINTER(Leaves64), C.POINTER(C.c_int32)]),
    "hmvm_b200_free_leaves64": (None, [C.POINTER(Leaves64)]),
    "hmvm_b200_convert_d2f": (C.c_int, [C.POINTER(Matrix_f), C.POINTER(Matrix2_f), C.POINTER(Matrix_d),
                                        C.POINTER(Matrix2_d)]),
    "hmvm_b200_free_matrix_d": (None, [C.POINTER(Matrix_d)]),
    "hmvm_b200_free_matrix_f": (None, [C.POINTER(Matrix_f)]),
    "hmvm_b200_free_matrix2_d": (None, [C.POINTER(Matrix2_d)]),
    "hmvm_b200_free_matrix2_f": (None, [C.POINTER(Matrix2_f)]),
    "hmvm_b200_default_opts": (None, [C.POINTER(PlanOpts)]),
    "hmvm_b200_plan_create_d": (C.c_int, [C.POINTER(Matrix2_d), C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "hmvm_b200_plan_create_f": (C.c_int, [C.POINTER(Matrix2_f), C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "hmvm_b200_plan_create64_d": (C.c_int, [C.POINTER(Leaves64), C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "hmvm_b200_plan_create64_f": (C.c_int, [C.POINTER(Leaves64), C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "hmvm_b200_plan_destroy": (None, [C.c_void_p]),
    "hmvm_b200_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    "hmvm_b200_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_apply_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_apply_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_cuda_d": (C.c_int, [C.POINTER(Matrix2_d), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(Stats)]),
    "hmvm_cuda_f": (C.c_int, [C.POINTER(Matrix2_f), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(Stats)]),
    "hmvm_b200_layout_build_d": (C.c_int, [C.POINTER(Matrix2_d), C.POINTER(PlanOpts), C.c_int32,
                                           C.POINTER(C.c_void_p)]),
    "hmvm_b200_layout_build64": (C.c_int, [C.POINTER(Leaves64), C.c_int32, C.POINTER(PlanOpts), C.c_int32,
                                           C.POINTER(C.c_void_p)]),
    "hmvm_b200_layout_view": (C.c_int, [C.c_void_p, C.POINTER(LayoutView)]),
    "hmvm_b200_layout_validate": (C.c_int, [C.c_void_p]),
    "hmvm_b200_plan_descriptors": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32)]),
    "hmvm_b200_layout_destroy": (None, [C.c_void_p]),
    "hmvm_b200_strerror": (C.c_char_p, [C.c_int]),
    "hmvm_b200_last_error": (C.c_char_p, []),
    "hmvm_b200_version": (C.c_int, []),
    "hmvm_b200_plan_kernel_count": (C.c_int, [C.c_void_p]),
    "hmvm_b200_apply_multi": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32,
                                        C.c_void_p]),
    "hmvm_b200_apply_multi_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32,
                                             C.c_void_p]),
    "hmvm_b200_plan_multi_kernel_count": (C.c_int, [C.c_void_p, C.c_int32]),
    "hmvm_b200_plan_capture": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_plan_replay": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hmvm_b200_bicgstab": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "hmvm_b200_gcrm": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "hmvm_b200_autotune64": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "hmvm_b200_autotune_d": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "hmvm_b200_shape_histogram64": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hmvm_b200_autotune_cached64": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_char_p, C.c_double,
                                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_create64_d": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_create64_f": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_create_d": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_destroy": (None, [C.c_void_p]),
    "hmvm_b200_batch_get_info": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_instance": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_class_count": (C.c_int, [C.c_void_p]),
    "hmvm_b200_batch_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "hmvm_b200_batch_capture": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    "hmvm_b200_batch_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "hmvm_b200_batch_status": (C.c_int, [C.c_void_p]),
    "hmvm_b200_batch_kernel_count": (C.c_int, [C.c_void_p]),
    "hmvm_b200_plan_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "hmvm_b200_plan_profile_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "hmvm_b200_plan_status": (C.c_int, [C.c_void_p]),
    "hmvm_b200_aca_fill": (C.c_int, [C.POINTER(HgenMatrix), C.POINTER(HgenParams), C.c_int32,
                                     C.POINTER(AcaReport)]),
}

HGEN_SIGNATURES = {
    "hgen_default_params": (None, [C.POINTER(HgenParams)]),
    "hgen_build": (C.c_int, [C.POINTER(HgenParams), C.POINTER(C.POINTER(HgenMatrix))]),
    "hgen_build_tree": (C.c_int, [C.POINTER(HgenParams), C.POINTER(C.POINTER(HgenMatrix))]),
    "hgen_build_tree_mesh": (C.c_int, [C.POINTER(HgenParams), C.POINTER(HgenMesh), C.POINTER(C.POINTER(HgenMatrix))]),
    "hgen_read_pbf": (C.c_int, [C.c_char_p, C.POINTER(C.POINTER(HgenMesh))]),
    "hgen_free_mesh": (None, [C.POINTER(HgenMesh)]),
    "hgen_fill_leaves": (C.c_int, [C.POINTER(HgenMatrix), C.POINTER(HgenParams)]),
    "hgen_free": (None, [C.POINTER(HgenMatrix)]),
    "hgen_write_bin1": (C.c_int, [C.POINTER(HgenMatrix), C.c_char_p]),
    "hgen_write_bin2": (C.c_int, [C.POINTER(HgenMatrix), C.c_char_p]),
    "hgen_write_bin64": (C.c_int, [C.POINTER(HgenMatrix), C.c_char_p]),
    "hgen_entry": (C.c_double, [C.POINTER(HgenMatrix), C.c_int32, C.c_int32]),
}

_hmvm = None
_hgen = None


def _bind(lib, sigs):
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def hmvm_lib():
    """The HMVM library; raises ImportError when it has not been built."""
    global _hmvm
    if _hmvm is None:
        if not os.path.exists(LIB_HMVM_PATH):
            raise ImportError(f"{LIB_HMVM_PATH} is missing: run `python -m hacapk_hmvm_b200.build`")
        _hmvm = _bind(C.CDLL(LIB_HMVM_PATH), HMVM_SIGNATURES)
    return _hmvm


def hgen_lib():
    global _hgen
    if _hgen is None:
        if not os.path.exists(LIB_HGEN_PATH):
            raise ImportError(f"{LIB_HGEN_PATH} is missing: run `python -m hacapk_hmvm_b200.build`")
        _hgen = _bind(C.CDLL(LIB_HGEN_PATH), HGEN_SIGNATURES)
    return _hgen


class HMVMError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = hmvm_lib()
        msg = lib.hmvm_b200_last_error().decode(errors="replace")
        name = lib.hmvm_b200_strerror(status).decode()
        super().__init__(f"{where}: {name} ({status}): {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != HMVM_OK:
        raise HMVMError(status, where)
