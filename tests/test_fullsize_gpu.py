"""Parity at the benchmark configurations' full sizes (the other GPU tests run
at N <= 16,384).

C1  sphere, N = 262,144, leaf 32, eta 2, ACA eps 1e-4, x uniform[-1, 1]
    (seeded), against the reference's own hmvm_omp_2<double,0> (oracle/_ref,
    src_hmvm/src_cpp/hmvm_omp.cpp:374-463) on the same FP64 elements:
      FP32 single vector                       <= 1e-5 (the FP32 bar)
      mixed single vector, FP16 factors         <= 1e-4 (the mixed bar)
      mixed 128 right-hand sides on the wide tensor-core form, 8 columns
      checked                                   <= 1e-4
      FP32 storage, 128 right-hand sides on the wide tensor-core form
                                                <= 1e-5
C2  cube surface, N = 1,048,576, leaf 32, eta 2, ACA eps 1e-4, x standard
    normal, mixed (FP16 factors) through the 64-bit leaf table (its element
    count exceeds the reference's int offsets), against the oracle's 64-bit
    restatement of hmvm_seq_2 / hmvm_omp_2 (oracle/hmvm_oracle.c, itself
    bitwise equal to the reference build where both run): <= 1e-4.

Each measured error is printed in the run's terminal summary beside its bound
and the ACA tolerance.
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from helpers import RefMatrix, oracle_omp, ref_available, relerr

pytestmark = pytest.mark.gpu

_C1 = {}


def _c1():
    if not _C1:
        hm = HMatrix.generate(262144, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=2024)
        X = np.random.default_rng(2024).uniform(-1.0, 1.0, (128, hm.nd))
        if ref_available():
            ref = RefMatrix(hm)
            ys = {c: ref.omp2(X[c]) for c in (0, 1, 31, 64, 90, 127, 100, 50)}
            kind = "reference hmvm_omp_2"
        else:
            ys = {c: oracle_omp(hm, X[c]) for c in (0, 1, 31, 64, 90, 127, 100, 50)}
            kind = "oracle port"
        _C1.update(hm=hm, X=X, ys=ys, kind=kind)
    return _C1


def _apply(plan, X):
    import torch

    dt = torch.float32 if plan.precision == "fp32" else torch.float64
    xd = torch.from_numpy(X).to(device="cuda", dtype=dt)
    yd = torch.full_like(xd, float("nan"))
    if X.shape[0] == 1:
        plan.apply(xd[0], yd[0])
    else:
        plan.apply_multi(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    return yd.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("prec,nrhs,tol", [("fp32", 1, 1e-5), ("mixed", 1, 1e-4), ("mixed", 128, 1e-4),
                                           ("fp32", 128, 1e-5)],
                         ids=["fp32", "mixed", "mixed-tc128", "fp32-tc128"])
def test_c1_parity(gpu, report, prec, nrhs, tol):
    c = _c1()
    hm, X, ys = c["hm"], c["X"], c["ys"]
    with Plan(hm, prec, nrhs_max=128 if nrhs > 1 else 1) as plan:
        Y = _apply(plan, X[:nrhs])
    cols = [k for k in ys if k < nrhs]
    err = max(relerr(Y[k], ys[k]) for k in cols)
    report.append(f"C1 sphere N=262144 {prec} nrhs={nrhs} ({len(cols)} columns) vs {c['kind']}: "
                  f"{err:.3e} (bound {tol:g}, ACA eps 1e-4)")
    assert err <= tol, err


def test_c2_parity(gpu, report):
    hm = HMatrix.generate(1048576, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=2024)
    assert not hm.fits_matrix2()  # beyond the reference's int offsets: the 64-bit leaf table
    x = np.random.default_rng(2024).standard_normal(hm.nd)
    y_or = oracle_omp(hm, x)
    with Plan(hm, "mixed") as plan:
        y = _apply(plan, x[None, :])[0]
    err = relerr(y, y_or)
    report.append(f"C2 cube N=1048576 mixed (64-bit leaf table) vs oracle 64-bit port: {err:.3e} "
                  f"(bound 1e-4, ACA eps 1e-4)")
    assert err <= 1e-4, err
