"""hmvm_b200_apply_noalloc: y = H x without allocating GPU memory.

Some callers may not call cudaMalloc while they run -- for example a solver
embedded in an application that hands out all device memory from its own pool,
or code with a device-memory budget fixed at start-up.  For them the library
keeps its HMVM scratch (the V x vector and split-panel partial sums) in one
fixed 16 MiB device array instead of per-plan buffers.  These tests call that
entry point through the C ABI and compare it with hmvm_b200_apply on the same
inputs, on consecutive calls that share (and inherit the contents of) the
array.  Both entry points run the same kernels in the same fixed order, so the
results must agree bit for bit (the tolerance the other GPU tests use for a
path against itself); the device's free memory must not move across the calls.
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan, _lib
from helpers import relerr

pytestmark = pytest.mark.gpu


def _bits(a):
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _dev(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _both(plan, x):
    """(hmvm_b200_apply result, hmvm_b200_apply_noalloc result, free device
    bytes before and after the no-alloc call) for one x."""
    import torch

    tdt = torch.float64 if plan.dtype == np.float64 else torch.float32
    xd = _dev(x, plan.dtype)
    y_ref = torch.full((plan.nd,), float("nan"), dtype=tdt, device="cuda")
    y_new = torch.full((plan.nd,), float("nan"), dtype=tdt, device="cuda")
    plan.apply(xd, y_ref)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    plan.apply_noalloc(xd, y_new)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return y_ref.cpu().numpy(), y_new.cpu().numpy(), free0, free1


def test_noalloc_matches_apply_on_consecutive_calls(gpu):
    # Two different H-matrices (different scratch layouts) and both precisions,
    # called back to back: each call starts from the previous call's leftovers.
    mats = [HMatrix.generate(3000, "cube", eps=1e-4, seed=21), HMatrix.generate(2048, "sphere", eps=1e-6, seed=22)]
    rng = np.random.default_rng(5)
    calls = 0
    for prec in ("fp64", "fp32"):
        for k, hm in enumerate(mats):
            # a small split width also routes some V panels through the partial sums
            with Plan(hm, prec, split_cols=64 if k == 0 else 0) as plan:
                for _ in range(2):
                    x = rng.uniform(-1.0, 1.0, hm.nd)
                    y_ref, y_new, free0, free1 = _both(plan, x)
                    assert np.all(np.isfinite(y_new))
                    assert np.array_equal(_bits(y_new), _bits(y_ref)), (prec, k, relerr(y_new, y_ref))
                    # the first call on the device may look the array up; later calls allocate nothing
                    if calls > 0:
                        assert free1 == free0, (prec, k, free0 - free1)
                    calls += 1
    assert calls == 8


def test_noalloc_rejects_plans_beyond_the_array(gpu):
    # One low-rank leaf of rank 2.2M on a 1x1 block: its V x vector alone needs
    # 17.6 MB of scratch, more than the 16 MiB array.
    kt = 2_200_000
    hm = HMatrix.from_arrays(1, kt, [1], [kt], [1], [1], [1], [1], [0], [kt], np.full(2 * kt, 0.5))
    import torch

    with Plan(hm, "fp64") as plan:
        assert plan.info()["t_len"] * 8 > _lib.HMVM_NOALLOC_SCRATCH_BYTES
        xd = torch.ones(1, dtype=torch.float64, device="cuda")
        yd = torch.zeros(1, dtype=torch.float64, device="cuda")
        with pytest.raises(_lib.HMVMError) as e:
            plan.apply_noalloc(xd, yd)
        assert e.value.status == _lib.HMVM_ERANGE
        assert "scratch" in str(e.value)
        plan.apply(xd, yd)  # the ordinary entry point still serves it
        torch.cuda.synchronize()
        assert yd.item() == pytest.approx(0.25 * kt, rel=1e-12)
