"""Tensor-core multi-RHS passes (mixed plans with nrhs_max = 16): the FP16/BF16
factor runs on tcgen05 (hmvm_tc_kernel), everything else on the CUDA cores.

Every column of Y against the FP64 oracle: relative error <= 1e-4 (the mixed
bar); and against the CUDA-core multi-RHS kernel on the same stored formats
(relative difference <= 2e-5: the tensor-core path adds only the 16-bit
hi/lo split of its inputs, about 2^-22 relative for FP16, 2^-17 for BF16).
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from helpers import oracle_hmvm, relerr

pytestmark = pytest.mark.gpu

_cache = {}


def _mat(n=3000, geo="cube", seed=2, eps=1e-4):
    key = (n, geo, seed, eps)
    if key not in _cache:
        _cache[key] = HMatrix.generate(n, geo, eta=2.0, eps=eps, leaf_size=32, seed=seed)
    return _cache[key]


def _run(plan, X):
    import torch

    xd = torch.from_numpy(X).cuda()
    yd = torch.full_like(xd, float("nan"))
    plan.apply_multi(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    return yd.cpu().numpy()


@pytest.mark.parametrize("fmt", ["fp16", "bf16"])
@pytest.mark.parametrize("case", [(3000, "cube", 2, 1e-4), (2048, "sphere", 1, 1e-6), (1500, "plate", 3, 1e-3)],
                         ids=lambda c: f"{c[1]}{c[0]}")
def test_tc_parity(gpu, fmt, case):
    hm = _mat(*case)
    X = np.random.default_rng(1).uniform(-1, 1, (20, hm.nd))
    with Plan(hm, "mixed", nrhs_max=16, mixed_lr_format=fmt) as tc, \
            Plan(hm, "mixed", nrhs_max=8, mixed_lr_format=fmt) as cc:
        assert tc.multi_kernel_count(20) == 2 * tc.multi_kernel_count(16)  # two 16-column passes
        Yt = _run(tc, X)
        Yc = _run(cc, X)
    for r in range(X.shape[0]):
        yo = oracle_hmvm(hm, X[r])
        assert relerr(Yt[r], yo) <= 1e-4, (r, relerr(Yt[r], yo))
        assert relerr(Yt[r], Yc[r]) <= 2e-5, (r, relerr(Yt[r], Yc[r]))


def test_tc_column_scales_and_ragged(gpu):
    """Columns of very different magnitude in one pass (each right-hand side
    has its own power-of-two scale in the 16-bit planes), a ragged pass of 5
    columns, and bitwise repeatability."""
    hm = _mat(2048, "sphere", 5)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((5, hm.nd)) * np.array([1e-12, 1.0, 1e6, 3e3, 1e-3])[:, None]
    with Plan(hm, "mixed", nrhs_max=16) as tc:
        Y1 = _run(tc, X)
        Y2 = _run(tc, X)
    assert np.array_equal(Y1, Y2)
    for r in range(5):
        assert relerr(Y1[r], oracle_hmvm(hm, X[r])) <= 1e-4, (r, relerr(Y1[r], oracle_hmvm(hm, X[r])))
