"""hacapk_hmvm_b200: H-matrix-vector multiplication on one NVIDIA B200.

A drop-in for the HMVM path of hacapk_hmvm: the same H-matrix structures and
hmatrix_1.bin / hmatrix_2.bin files, computed by hand-written sm_100a kernels
behind the C ABI in include/hmvm_b200.h.
"""
from .hmatrix import HMatrix  # noqa: F401
from .hmvm import Plan, autotune, hmvm, hmvm_cuda  # noqa: F401
from .batch import Batch  # noqa: F401

__all__ = ["HMatrix", "Plan", "Batch", "autotune", "hmvm", "hmvm_cuda"]
