"""Wide tensor-core multi-RHS passes (FP32 and mixed plans made with
nrhs_max >= 32): 128 right-hand sides per pass, every product on tcgen05
(hmvm_tcw_kernel).

Each checked column of Y against
  * the FP64 oracle (the reference's hmvm_seq_2 arithmetic): relative error
    <= 1e-4 for mixed plans (the mixed bar) and <= 1e-5 for FP32 plans (the
    FP32 bar; the pairs hold about 22 significant bits);
  * a CPU walk of the very same layout (tests/helpers.py:emulate_tcw), which
    sums in FP64 where the tensor cores accumulate in FP32: relative
    difference <= 1e-5 (a layout or indexing fault shows as O(1)).
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from hacapk_hmvm_b200.hmvm import PRECISIONS
from helpers import emulate_tcw, layout_for, oracle_hmvm, relerr

pytestmark = pytest.mark.gpu

TOL_ORACLE = {"mixed": 1e-4, "fp32": 1e-5}
TOL_EMU = {"mixed": 1e-5, "fp32": 1e-5}
_cache = {}


def _mat(n, geo, seed, eps=1e-4):
    key = (n, geo, seed, eps)
    if key not in _cache:
        _cache[key] = HMatrix.generate(n, geo, eta=2.0, eps=eps, leaf_size=32, seed=seed)
    return _cache[key]


def _run(plan, X):
    import torch

    dt = torch.float32 if plan.precision == "fp32" else torch.float64
    xd = torch.from_numpy(X).to(device="cuda", dtype=dt)
    yd = torch.full_like(xd, float("nan"))
    plan.apply_multi(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    return yd.cpu().numpy().astype(np.float64)


def _check(hm, prec, fmt, X, Y, cols):
    kw = dict(precision=PRECISIONS[prec], nrhs_max=128)
    if fmt:
        kw["mixed_lr_format"] = fmt
    _, view = layout_for(hm, **kw)
    assert view.tcw == 1
    Xc = X.astype(np.float32).astype(np.float64) if prec == "fp32" else X
    for c0 in range(0, X.shape[0], 128):
        blk = [c for c in cols if c0 <= c < c0 + 128]
        if not blk:
            continue
        E = emulate_tcw(view, Xc[c0:c0 + 128])
        for c in blk:
            yo = oracle_hmvm(hm, X[c])
            assert np.all(np.isfinite(Y[c])), c
            assert relerr(Y[c], yo) <= TOL_ORACLE[prec], (c, relerr(Y[c], yo))
            assert relerr(Y[c], E[c - c0]) <= TOL_EMU[prec], (c, relerr(Y[c], E[c - c0]))


@pytest.mark.parametrize("prec,fmt", [("mixed", "fp16"), ("mixed", "bf16"), ("fp32", None)])
# N (= the leading dimension of Y) sets the row stage's stores: multiples of 4 take
# 16-byte stores for FP64 and FP32 outputs, 1202 for FP64 only, 1201 single stores.
@pytest.mark.parametrize("case", [(3000, "cube", 2), (2048, "sphere", 1), (1500, "plate", 3), (1202, "sphere", 4),
                                  (1201, "cube", 6)],
                         ids=lambda c: f"{c[1]}{c[0]}")
def test_tcw_parity(gpu, prec, fmt, case):
    hm = _mat(*case)
    X = np.random.default_rng(1).uniform(-1, 1, (40, hm.nd))
    with Plan(hm, prec, nrhs_max=128, mixed_lr_format=fmt) as plan:
        assert plan.info()["kernel"] == 4
        Y = _run(plan, X)
    _check(hm, prec, fmt, X, Y, range(40))


@pytest.mark.parametrize("prec,fmt", [("mixed", "fp16"), ("fp32", None)])
def test_tcw_split_panels_and_two_passes(gpu, prec, fmt):
    """A matrix whose V-stage panels are cut into parts (FP32 partial sums
    added by hmvm_tcw_reduce_kernel), 130 right-hand sides (a full pass and
    a ragged one), columns of very different magnitude, bitwise repeatable."""
    hm = _mat(16384, "sphere", 5)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((130, hm.nd)) * np.exp(rng.uniform(-8, 8, 130))[:, None]
    with Plan(hm, prec, nrhs_max=128, mixed_lr_format=fmt) as plan:
        assert plan.info()["split_rows"] > 0
        assert plan.multi_kernel_count(130) == 2 * plan.multi_kernel_count(128)
        Y1 = _run(plan, X)
        Y2 = _run(plan, X)
    assert np.array_equal(Y1, Y2)
    _check(hm, prec, fmt, X, Y1, [0, 1, 63, 64, 127, 128, 129])


def test_tcw_single_vector_apply(gpu):
    """apply() on a wide tensor-core plan runs one pass with one column."""
    import torch

    hm = _mat(2048, "sphere", 1)
    x = np.sin(np.arange(1, hm.nd + 1, dtype=np.float64))
    with Plan(hm, "mixed", nrhs_max=128) as plan:
        xd = torch.from_numpy(x).cuda()
        yd = torch.full_like(xd, float("nan"))
        plan.apply(xd, yd)
        torch.cuda.synchronize()
        plan.status()
    assert relerr(yd.cpu().numpy(), oracle_hmvm(hm, x)) <= 1e-4
