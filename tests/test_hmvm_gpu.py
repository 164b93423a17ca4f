"""Parity of the sm_100a HMVM against the oracle (hmvm_seq_2<double,0>
restated, pinned to the reference) and the reference's own build, through the
C ABI.

Tolerances (relative 2-norm error against the FP64 oracle):
  FP64 plans  <= 1e-12
  FP32 plans  <= 1e-5
"""
import ctypes as C

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan, _lib, hmvm
from helpers import RefMatrix, oracle_hmvm, ref_available, relerr

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5

CASES = [
    # n, geometry, eta, eps, leaf, seed
    (2048, "sphere", 2.0, 1e-4, 32, 1),
    (3000, "cube", 2.0, 1e-4, 32, 2),
    (1200, "plate", 1.0, 1e-6, 32, 3),
    (1000, "sphere", 2.0, 1e-3, 8, 4),     # small leaves: many tiny tiles
    (777, "cube", 1.0, 1e-4, 45, 5),       # leaf > 32 rows: finest intervals split
    (8192, "sphere", 2.0, 1e-4, 32, 7),    # the N=8,192 sphere of the CPU configuration
]

_cache = {}


def _mat(case):
    if case not in _cache:
        n, geo, eta, eps, leaf, seed = case
        _cache[case] = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=seed)
    return _cache[case]


def _x(n, kind="uniform", seed=0):
    if kind == "sin":
        return np.sin(np.arange(1, n + 1, dtype=np.float64))  # hmvm1.cpp:37-41
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def _run(plan, x):
    import torch

    dt = torch.float64 if plan.dtype == np.float64 else torch.float32
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=plan.dtype)).cuda()
    yd = torch.full((plan.nd,), float("nan"), dtype=dt, device="cuda")
    plan.apply(xd, yd)
    torch.cuda.synchronize()
    plan.status()  # raises if a kernel gave up on a bounded wait
    return yd.cpu().numpy()


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[1]}{c[0]}_eta{c[2]}_eps{c[3]}_leaf{c[4]}")
def test_fp64_parity(gpu, case):
    hm = _mat(case)
    for kind in ("sin", "uniform"):
        x = _x(hm.nd, kind)
        yo = oracle_hmvm(hm, x)
        with Plan(hm, "fp64") as plan:
            y = _run(plan, x)
        assert np.all(np.isfinite(y))
        assert relerr(y, yo) <= TOL64, (kind, relerr(y, yo))
        if ref_available():
            yr = RefMatrix(hm).seq2(x)
            assert relerr(y, yr) <= TOL64


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[1]}{c[0]}_eta{c[2]}_eps{c[3]}_leaf{c[4]}")
def test_fp32_parity(gpu, case):
    hm = _mat(case)
    x = _x(hm.nd, "uniform", seed=1)
    yo = oracle_hmvm(hm, x)  # FP64 oracle
    # FP32 plan built from the double matrix (elements rounded as convertD2F)
    with Plan(hm, "fp32") as plan:
        y = _run(plan, x)
    assert relerr(y, yo) <= TOL32, relerr(y, yo)
    # and from an explicitly converted float matrix, against the float reference
    hf = hm.to_float()
    with Plan(hf, "fp32") as plan:
        y2 = _run(plan, x)
    np.testing.assert_array_equal(y, y2)
    yf = oracle_hmvm(hf, x.astype(np.float32))
    assert relerr(y2, yf) <= TOL32
    if ref_available():
        yr = RefMatrix(hm).seq2_f(x.astype(np.float32))
        assert relerr(y2, yr) <= TOL32


def test_bitwise_repeatable(gpu):
    hm = _mat(CASES[0])
    x = _x(hm.nd)
    with Plan(hm, "fp64") as plan:
        ys = [_run(plan, x) for _ in range(3)]
    for y in ys[1:]:
        assert np.array_equal(y.view(np.uint64), ys[0].view(np.uint64))


NCFGS = {0: 8, 1: 8}  # kNumCfgs, kNumStreamCfgs (layout.hpp)
KCFGS = [(k, c) for k in (0, 1) for c in range(NCFGS[k])]


@pytest.mark.parametrize("kernel,cfg1", KCFGS, ids=[f"k{k}c{c}" for k, c in KCFGS])
def test_kernel_configs(gpu, kernel, cfg1):
    """Both kernel variants, every configuration (team shape / ring shape),
    compute the same y within tolerance, in FP64 and FP32."""
    hm = _mat(CASES[1])
    x = _x(hm.nd)
    yo = oracle_hmvm(hm, x)
    ncfg = NCFGS[kernel]
    for prec, tol in (("fp64", TOL64), ("fp32", TOL32)):
        with Plan(hm, prec, kernel=kernel, stage1_cfg=cfg1, stage2_cfg=ncfg - 1 - cfg1,
                  ctas_per_sm=1 + cfg1 % 2) as plan:
            assert plan.info()["kernel"] == kernel
            y = _run(plan, x)
        assert relerr(y, yo) <= tol


def test_variants_agree(gpu):
    """The register-streaming and TMA-ring kernels walk the same layout."""
    hm = _mat(CASES[5])
    x = _x(hm.nd, "sin")
    ys = []
    for kernel in (0, 1):
        with Plan(hm, "fp64", kernel=kernel) as plan:
            ys.append(_run(plan, x))
    assert relerr(ys[0], ys[1]) <= TOL64


@pytest.mark.parametrize("split", [2, 8, 40, 1000])
def test_split_panels(gpu, split):
    """Wide V panels cut into column chunks and reduced in chunk order."""
    hm = _mat(CASES[0])
    x = _x(hm.nd)
    yo = oracle_hmvm(hm, x)
    for prec, tol in (("fp64", TOL64), ("fp32", TOL32)):
        with Plan(hm, prec, split_cols=split) as plan:
            if split < 1000:
                assert plan.info()["split_rows"] > 0
            y = _run(plan, x)
        assert relerr(y, yo) <= tol


@pytest.mark.parametrize("rows", [1, 7, 16, 31])
def test_tile_rows(gpu, rows):
    hm = _mat(CASES[3])
    x = _x(hm.nd)
    yo = oracle_hmvm(hm, x)
    with Plan(hm, "fp64", max_tile_rows=rows) as plan:
        y = _run(plan, x)
    assert relerr(y, yo) <= TOL64


def test_apply_host_and_one_shot(gpu):
    hm = _mat(CASES[2])
    x = _x(hm.nd, "sin")
    yo = oracle_hmvm(hm, x)
    with Plan(hm, "fp64") as plan:
        y1 = plan.apply_host(x)
        y2 = _run(plan, x)
    assert np.array_equal(y1, y2)
    y3, st = hmvm(hm, x)
    assert np.array_equal(y3, y1)
    assert st["seconds_apply"] > 0 and st["algorithmic_bytes"] == hm.algorithmic_bytes()
    y4, _ = hmvm(hm.to_float(), x)
    assert relerr(y4, yo) <= TOL32


def _kat_matrix():
    """Hand-built 6x6 leaf list: a rank-2 leaf, a rank-0 leaf, dense leaves, a
    1x1 dense leaf; small integer entries so y is exact."""
    leaves = []  # (ltmtx, ndl, ndt, nstrtl, nstrtt, kt, data)
    D1 = np.arange(1, 10, dtype=np.float64).reshape(3, 3)           # rows 1-3, cols 1-3
    V = np.array([[1, 0, 2], [0, 1, 1]], dtype=np.float64)          # kt=2, ndt=3 (cols 4-6)
    U = np.array([[1, 2, 3], [1, -1, 0]], dtype=np.float64)         # kt=2, ndl=3 (rows 1-3)
    D2 = np.array([[2, 0], [0, 3]], dtype=np.float64)               # rows 4-5, cols 4-5
    leaves.append((2, 3, 3, 1, 1, 0, D1.ravel()))
    leaves.append((1, 3, 3, 1, 4, 2, np.concatenate([V.ravel(), U.ravel()])))
    leaves.append((1, 3, 3, 4, 1, 0, np.zeros(0)))                  # kt = 0: contributes nothing
    leaves.append((2, 2, 2, 4, 4, 0, D2.ravel()))
    leaves.append((2, 2, 1, 4, 6, 0, np.array([1.0, -1.0])))        # rows 4-5, col 6
    leaves.append((2, 1, 2, 6, 4, 0, np.array([5.0, 7.0])))         # row 6, cols 4-5
    leaves.append((2, 1, 1, 6, 6, 0, np.array([-4.0])))             # row 6, col 6
    a1, a2, data, off = [], [], [], 0
    for lt, ndl, ndt, sl, st, kt, d in leaves:
        if lt == 1:
            a1.append(off)
            a2.append(off + kt * ndt)
        else:
            a1.append(off)
            a2.append(0)
        data.append(d)
        off += d.size
    A = np.zeros((6, 6))
    A[0:3, 0:3] = D1
    A[0:3, 3:6] = U.T @ V
    A[3:5, 3:5] = D2
    A[3:5, 5] = [1, -1]
    A[5, 3:5] = [5, 7]
    A[5, 5] = -4
    hm = HMatrix.from_arrays(6, 2, [l[0] for l in leaves], [l[5] for l in leaves], [l[1] for l in leaves],
                             [l[2] for l in leaves], [l[3] for l in leaves], [l[4] for l in leaves], a1, a2,
                             np.concatenate(data))
    return hm, A


def test_known_answer(gpu):
    hm, A = _kat_matrix()
    x = np.array([1.0, -2.0, 3.0, 0.5, -1.5, 2.0])
    yexact = A @ x
    assert np.array_equal(oracle_hmvm(hm, x), yexact)
    for prec in ("fp64", "fp32"):
        with Plan(hm, prec) as plan:
            y = _run(plan, x)
        assert np.array_equal(y.astype(np.float64), yexact), (prec, y, yexact)


def test_uncovered_rows_are_zero(gpu):
    """Rows no leaf touches come out as 0 (y is overwritten, not accumulated)."""
    hm = HMatrix.from_arrays(5, 1, [2], [0], [2], [2], [2], [1], [0], [0], np.array([1.0, 2.0, 3.0, 4.0]))
    x = np.arange(1.0, 6.0)
    with Plan(hm, "fp64") as plan:
        y = _run(plan, x)
    assert np.array_equal(y, [0.0, 1 * 1 + 2 * 2, 3 * 1 + 4 * 2, 0.0, 0.0])


def test_empty_and_single(gpu):
    hm0 = HMatrix.from_arrays(0, 0, [], [], [], [], [], [], [], [], np.zeros(0))
    with Plan(hm0, "fp64") as plan:
        assert plan.kernel_count() == 0
    hm1 = HMatrix.from_arrays(1, 0, [2], [0], [1], [1], [1], [1], [0], [0], np.array([3.5]))
    with Plan(hm1, "fp64") as plan:
        assert _run(plan, np.array([2.0]))[0] == 7.0


def test_invalid_tables_rejected(gpu):
    hm, _ = _kat_matrix()
    bad = HMatrix.from_arrays(hm.nd, hm.ktmax, hm.ltmtx, hm.kt, hm.ndl, hm.ndt, hm.nstrtl, hm.nstrtt, hm.a1,
                              hm.a2, hm.rowmat)
    bad.kt[1] = 5  # > ktmax
    with pytest.raises(_lib.HMVMError) as e:
        Plan(bad, "fp64")
    assert e.value.status == _lib.HMVM_EINVAL


def test_overlapping_xy_rejected(gpu):
    import torch

    hm = _mat(CASES[3])
    with Plan(hm, "fp64") as plan:
        buf = torch.zeros(hm.nd + 10, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.HMVMError):
            plan.apply(buf.data_ptr(), buf.data_ptr() + 8 * 5)


def test_streams(gpu):
    """Launches go to the given stream; results match the default stream's."""
    import torch

    hm = _mat(CASES[0])
    x = _x(hm.nd)
    with Plan(hm, "fp64") as plan:
        y0 = _run(plan, x)
        s = torch.cuda.Stream()
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            plan.apply(xd, yd, stream=s)
        s.synchronize()
        assert np.array_equal(yd.cpu().numpy(), y0)


def test_golden_fixtures(gpu):
    """The committed fixtures: inputs as bytes, y from the reference's own hmvm_seq_2."""
    import json
    import os

    from helpers import GOLDEN

    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))
    Y = np.load(os.path.join(GOLDEN, "golden_y.npz"))
    for name, m in meta["matrices"].items():
        hm = HMatrix.load(os.path.join(GOLDEN, m["file"]))
        for xn in ("sin", "uniform"):
            x = Y[f"{name}/x_{xn}"]
            with Plan(hm, "fp64") as plan:
                y = _run(plan, x)
            assert relerr(y, Y[f"{name}/y_seq2_d_{xn}"]) <= TOL64, (name, xn)
            with Plan(hm, "fp32") as plan:
                yf = _run(plan, x)
            assert relerr(yf, Y[f"{name}/y_seq2_f_{xn}"]) <= TOL32, (name, xn)
            assert relerr(yf, Y[f"{name}/y_seq2_d_{xn}"]) <= TOL32


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_capture_replay(gpu, prec):
    """hmvm_b200_plan_capture + hmvm_b200_plan_replay: a replayed graph of one
    apply gives y bit for bit equal to the direct apply, follows new contents
    of x, and a new capture replaces the old one."""
    import torch

    from hacapk_hmvm_b200 import _lib

    hm = HMatrix.generate(3000, "sphere", eta=2.0, eps=1e-5, leaf_size=24, seed=6)
    dt = torch.float32 if prec == "fp32" else torch.float64
    with Plan(hm, prec) as plan:
        with pytest.raises(_lib.HMVMError):
            plan.replay()  # nothing captured yet
        x = torch.rand(hm.nd, dtype=dt, device="cuda") - 0.5
        y_ref, y = torch.empty_like(x), torch.full_like(x, float("nan"))
        plan.apply(x, y_ref)
        plan.capture(x, y)
        for _ in range(2):
            plan.replay()
            torch.cuda.synchronize()
            assert torch.equal(y, y_ref)
        x.mul_(-2.0)  # the graph reads the buffer's current contents
        plan.apply(x, y_ref)
        plan.replay()
        torch.cuda.synchronize()
        assert torch.equal(y, y_ref)
        x2, y2 = torch.rand_like(x), torch.empty_like(x)
        plan.capture(x2, y2)
        plan.replay()
        plan.apply(x2, y_ref)
        torch.cuda.synchronize()
        assert torch.equal(y2, y_ref)
        plan.profile(True)
        with pytest.raises(_lib.HMVMError):
            plan.capture(x, y)
        plan.profile(False)
