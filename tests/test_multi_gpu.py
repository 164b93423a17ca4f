"""Multi-RHS HMVM (hmvm_b200_apply_multi) on the GPU, through the C ABI.

Every column of Y is checked against the FP64 oracle applied to that column
of X, with the single-vector bars: FP64 plans <= 1e-12, FP32 plans <= 1e-5,
mixed plans <= 1e-4 (relative 2-norm error per column).  Column blocks run
in passes of up to nrhs_max columns; ragged last passes, leading dimensions
above N and host buffers are covered.
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from helpers import oracle_hmvm, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5, "mixed": 1e-4}
_cache = {}


def _mat(n=3000, geo="cube", seed=2):
    key = (n, geo, seed)
    if key not in _cache:
        _cache[key] = HMatrix.generate(n, geo, eta=2.0, eps=1e-4, leaf_size=32, seed=seed)
    return _cache[key]


def _oracle_cols(hm, X):
    return np.stack([oracle_hmvm(hm, X[r]) for r in range(X.shape[0])])


def _run(plan, X, ldx=None, ldy=None):
    import torch

    nrhs, n = X.shape
    ldx = ldx or n
    ldy = ldy or n
    dt = torch.float32 if plan.dtype == np.float32 else torch.float64
    xb = torch.zeros((nrhs, ldx), dtype=dt, device="cuda")
    xb[:, :n] = torch.from_numpy(X.astype(plan.dtype))
    yb = torch.full((nrhs, ldy), float("nan"), dtype=dt, device="cuda")
    plan.apply_multi(xb[:, :n], yb[:, :n])
    torch.cuda.synchronize()
    plan.status()
    Y = yb.cpu().numpy()
    if ldy > n:
        assert np.all(np.isnan(Y[:, n:])), "writes past N in a column"
    return Y[:, :n].astype(np.float64)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("nrhs_max", [2, 4, 8])
def test_multi_parity(gpu, prec, nrhs_max):
    hm = _mat()
    rng = np.random.default_rng(nrhs_max)
    X = rng.uniform(-1, 1, (13, hm.nd))
    Yo = _oracle_cols(hm, X)
    with Plan(hm, prec, nrhs_max=nrhs_max) as plan:
        for nrhs in (1, 2, 3, 8, 13):
            Y = _run(plan, X[:nrhs])
            for r in range(nrhs):
                assert relerr(Y[r], Yo[r]) <= TOL[prec], (nrhs, r, relerr(Y[r], Yo[r]))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_multi_leading_dimensions_and_host(gpu, prec):
    hm = _mat(2048, "sphere", 1)
    X = np.random.default_rng(7).uniform(-1, 1, (6, hm.nd))
    Yo = _oracle_cols(hm, X)
    with Plan(hm, prec, nrhs_max=4, split_cols=64) as plan:
        Y = _run(plan, X, ldx=hm.nd + 5, ldy=hm.nd + 3)
        Yh = plan.apply_multi_host(X)
        Y2 = _run(plan, X)
    for r in range(6):
        assert relerr(Y[r], Yo[r]) <= TOL[prec]
    assert np.array_equal(Yh, Y2) and np.array_equal(Y, Y2)  # fixed summation order


def test_multi_on_single_vector_plan(gpu):
    """nrhs_max = 1: columns run as single-vector applies, bit-identical to apply."""
    import torch

    hm = _mat(1500, "plate", 3)
    X = np.random.default_rng(2).uniform(-1, 1, (3, hm.nd))
    with Plan(hm, "fp64") as plan:
        Y = _run(plan, X)
        for r in range(3):
            xd = torch.from_numpy(X[r]).cuda()
            yd = torch.empty_like(xd)
            plan.apply(xd, yd)
            assert np.array_equal(yd.cpu().numpy(), Y[r])
        assert plan.multi_kernel_count(3) == 3 * plan.kernel_count()


def test_multi_repeatable_and_counts(gpu):
    hm = _mat()
    X = np.random.default_rng(5).uniform(-1, 1, (11, hm.nd))
    with Plan(hm, "mixed", nrhs_max=8) as plan:
        a, b = _run(plan, X), _run(plan, X)
        assert np.array_equal(a, b)
        # passes of 8, 2 and a lone column in a 2-wide pass
        assert plan.multi_kernel_count(11) == 3 * plan.multi_kernel_count(8)
