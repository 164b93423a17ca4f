"""The reference's own hybrid2 CUDA kernels (src_hmvm/src_cpp/hmvm_cuda2.cu,
built unchanged for sm_100a into oracle/_ref by oracle/Makefile), the same-box
GPU reference point bench.py times.  Test infrastructure: nothing in the
product links them.

Their y against the reference's hmvm_seq_2 (relative error <= 1e-12 in FP64,
<= 1e-5 in FP32; the kernels add with atomics, so only the summation order
differs), and the reference wrapper's own TIME line parses.  The variants are
the reference's fastest published ones (div 4, mul 12/13) and its default
shape; div 8/16 with a2i = 1, aa = 1, which the reference itself reports as
wrong (hmvm_cuda1.cu:391-392), are not used.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix
from helpers import ROOT, RefMatrix, oracle_hmvm, ref_available, relerr

pytestmark = pytest.mark.gpu

REF_CUDA_SO = os.path.join(ROOT, "oracle", "_ref", "libhmvm_ref_cuda.so")


def _libs(hm):
    if not (ref_available() and os.path.exists(REF_CUDA_SO)):
        pytest.skip("the reference build is not present")
    P = C.c_void_p
    ref = RefMatrix(hm)
    cuda = C.CDLL(REF_CUDA_SO)
    cuda.refgpu_cuda2_bench.argtypes = [P, C.c_int, P, C.c_int, C.c_int, C.c_char_p]
    cuda.refgpu_hybrid2_y.argtypes = [P, C.c_int, P] + [C.c_int] * 6 + [P]
    ref.lib.ref_matrix2_d.restype = P
    ref.lib.ref_matrix2_f.restype = P
    ref.lib.ref_matrix2_d.argtypes = [P]
    ref.lib.ref_matrix2_f.argtypes = [P]
    ref.lib.ref_make_float.argtypes = [P]
    return ref, cuda


@pytest.mark.parametrize("knobs", [(4, 12, 1, 1, 0, 0), (4, 13, 0, 1, 0, 0), (1, 1, 0, 0, 0, 0), (32, 2, 1, 0, 1, 1)],
                         ids=lambda k: "div%d_mul%d_a2t%d_a2i%d_aa%d_da%d" % k)
def test_reference_hybrid2_matches_oracle(gpu, knobs):
    hm = HMatrix.generate(4096, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=12)
    ref, cuda = _libs(hm)
    x = np.random.default_rng(4).uniform(-1, 1, hm.nd)
    y_or = oracle_hmvm(hm, x)
    y = np.empty(hm.nd)
    assert cuda.refgpu_hybrid2_y(ref.lib.ref_matrix2_d(ref.h), 0, x.ctypes.data, *knobs, y.ctypes.data) == 0
    assert relerr(y, y_or) <= 1e-12, relerr(y, y_or)
    assert ref.lib.ref_make_float(ref.h) == 0
    xf = x.astype(np.float32)
    yf = np.empty(hm.nd, np.float32)
    assert cuda.refgpu_hybrid2_y(ref.lib.ref_matrix2_f(ref.h), 1, xf.ctypes.data, *knobs, yf.ctypes.data) == 0
    assert relerr(yf, y_or) <= 1e-5, relerr(yf, y_or)


def test_reference_wrapper_time_line(gpu):
    hm = HMatrix.generate(2048, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=13)
    ref, cuda = _libs(hm)
    x = np.sin(np.arange(1, hm.nd + 1, dtype=np.float64))
    with tempfile.NamedTemporaryFile("r", suffix=".txt") as f:
        assert cuda.refgpu_cuda2_bench(ref.lib.ref_matrix2_d(ref.h), 0, x.ctypes.data, 356, 3, f.name.encode()) == 0
        lines = [ln.split() for ln in open(f.name) if ln.startswith("TIME")]
    assert len(lines) == 1 and lines[0][2] == "hmvm_cuda_hybrid2_div4_mul12_a2t1_a2i1_aa0_da0_d"
    tmin, tmax, tavg = float(lines[0][4]), float(lines[0][6]), float(lines[0][8])
    assert 0 < tmin <= tavg <= tmax
