"""Mixed-precision plans (HMVM_MIXED) on the GPU, through the C ABI.

Storage: low-rank columns in FP32 (leading terms), FP16 or BF16 (with
per-column scales), FP8 E4M3 (terms below eps * |block|); dense leaves FP32,
diagonal near-field blocks FP64; x and y in FP64.

Tolerances (relative 2-norm error):
  against the FP64 oracle                          <= 1e-4
  against the CPU walk of the same stored formats  <= 2e-6  (the kernels sum
      each segment in FP32, the CPU walk in FP64; this bound checks that the
      device decodes every format exactly as the planner stored it)
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan, _lib
from helpers import emulate_layout, layout_for, oracle_hmvm, relerr

pytestmark = pytest.mark.gpu

TOL_ORACLE = 1e-4
TOL_WALK = 2e-6

CASES = [
    (2048, "sphere", 2.0, 1e-4, 32, 1),
    (3000, "cube", 2.0, 1e-4, 32, 2),
    (1200, "plate", 1.0, 1e-6, 32, 3),
    (1000, "sphere", 2.0, 1e-3, 8, 4),
    (777, "cube", 1.0, 1e-4, 45, 5),
    (8192, "sphere", 2.0, 1e-4, 32, 7),
]

_cache = {}


def _mat(case):
    if case not in _cache:
        n, geo, eta, eps, leaf, seed = case
        _cache[case] = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=seed)
    return _cache[case]


def _x(n, seed=0):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def _run(plan, x):
    import torch

    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    yd = torch.full((plan.nd,), float("nan"), dtype=torch.float64, device="cuda")
    plan.apply(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    return yd.cpu().numpy()


def _walk(hm, x, **opts):
    h, v = layout_for(hm, precision=2, **opts)
    try:
        return emulate_layout(v, x)
    finally:
        _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[1]}{c[0]}_eta{c[2]}_eps{c[3]}_leaf{c[4]}")
def test_mixed_parity(gpu, case):
    hm = _mat(case)
    x = _x(hm.nd)
    yo = oracle_hmvm(hm, x)
    with Plan(hm, "mixed") as plan:
        info = plan.info()
        assert info["kernel"] == 2 and info["precision"] == _lib.HMVM_MIXED
        y = _run(plan, x)
    assert np.all(np.isfinite(y))
    assert relerr(y, yo) <= TOL_ORACLE, relerr(y, yo)
    assert relerr(y, _walk(hm, x)) <= TOL_WALK, relerr(y, _walk(hm, x))
    live = int(sum(k for k, t, l, c in zip(hm.kt, hm.ltmtx, hm.ndl, hm.ndt) if t == 1 and l > 0 and c > 0))
    assert info["cols_fp32"] + info["cols_lr16"] + info["cols_fp8"] == live


FORMAT_OPTS = [dict(mixed_lr_format="bf16"), dict(mixed_fp8_eps=0.0), dict(mixed_fp8_eps=1e-3),
               dict(mixed_fp32_tau=2.0), dict(mixed_fp32_tau=0.0)]


@pytest.mark.parametrize("opts", FORMAT_OPTS, ids=lambda o: "_".join(f"{k}={v}" for k, v in o.items()))
def test_mixed_formats(gpu, opts):
    """Every storage format decodes on the device as the planner stored it."""
    hm = _mat(CASES[2])
    x = _x(hm.nd, 3)
    with Plan(hm, "mixed", **opts) as plan:
        y = _run(plan, x)
    assert relerr(y, _walk(hm, x, **opts)) <= TOL_WALK
    assert relerr(y, oracle_hmvm(hm, x)) <= (2e-4 if opts.get("mixed_fp8_eps") == 1e-3 else TOL_ORACLE)


@pytest.mark.parametrize("cfg", range(11))
def test_mixed_kernel_configs(gpu, cfg):
    hm = _mat(CASES[1])
    x = _x(hm.nd, 1)
    opts = dict(stage1_cfg=cfg, stage2_cfg=10 - cfg, ctas_per_sm=1 + cfg % 2)
    with Plan(hm, "mixed", **opts) as plan:
        y = _run(plan, x)
    assert relerr(y, _walk(hm, x, **opts)) <= TOL_WALK
    assert relerr(y, oracle_hmvm(hm, x)) <= TOL_ORACLE


@pytest.mark.parametrize("opts", [dict(split_cols=8), dict(split_cols=40), dict(max_tile_rows=7)],
                         ids=["split8", "split40", "rows7"])
def test_mixed_split_and_rows(gpu, opts):
    hm = _mat(CASES[0])
    x = _x(hm.nd, 2)
    with Plan(hm, "mixed", **opts) as plan:
        if "split_cols" in opts:
            assert plan.info()["split_rows"] > 0
        y = _run(plan, x)
    assert relerr(y, _walk(hm, x, **opts)) <= TOL_WALK
    assert relerr(y, oracle_hmvm(hm, x)) <= TOL_ORACLE


def test_mixed_repeatable_host_and_noalloc(gpu):
    """Bitwise-identical repeats; apply_host and apply_noalloc give the same y."""
    import torch

    hm = _mat(CASES[5])
    x = _x(hm.nd, 4)
    with Plan(hm, "mixed", split_cols=64) as plan:
        ys = [_run(plan, x) for _ in range(3)]
        yh = plan.apply_host(x)
        xd = torch.from_numpy(x).cuda()
        yn = torch.full((hm.nd,), float("nan"), dtype=torch.float64, device="cuda")
        plan.apply_noalloc(xd, yn)
        torch.cuda.synchronize()
        yn = yn.cpu().numpy()
    for y in ys[1:] + [yh, yn]:
        assert np.array_equal(y.view(np.uint64), ys[0].view(np.uint64))


def test_mixed_stores_fewer_bytes(gpu):
    hm = _mat(CASES[5])
    with Plan(hm, "fp64") as p64, Plan(hm, "mixed") as pm:
        b64, bm = p64.info()["algorithmic_bytes"], pm.info()["algorithmic_bytes"]
    assert bm < 0.6 * b64, (bm, b64)
