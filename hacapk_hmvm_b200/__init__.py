"""hacapk_hmvm_b200: H-matrix-vector multiplication on one NVIDIA B200.

A drop-in for the HMVM path of hacapk_hmvm: the same H-matrix structures and
hmatrix_1.bin / hmatrix_2.bin files, computed by hand-written sm_100a kernels
behind the C ABI in include/hmvm_b200.h.
"""
from .hmatrix import HMatrix  # noqa: F401
from .hmvm import Plan, autotune, autotune_cached, hmvm, hmvm_cuda, shape_histogram  # noqa: F401
from .batch import Batch  # noqa: F401

__all__ = ["HMatrix", "Plan", "Batch", "autotune", "autotune_cached", "shape_histogram", "hmvm", "hmvm_cuda"]
