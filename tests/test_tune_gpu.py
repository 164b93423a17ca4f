"""The autotuner (hmvm_b200_autotune64): it times every candidate
configuration of both stages on the device, returns the options of the fastest
measured plan, and a plan built with them still meets the parity bars
(FP64 <= 1e-12, mixed <= 1e-4 against the FP64 oracle).  Through its cache
(hmvm_b200_autotune_cached64) a later matrix of the same family reuses the
stored choice without a sweep, with parity unchanged."""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan, autotune, autotune_cached
from helpers import oracle_hmvm, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-4)])
def test_autotune_picks_a_measured_best(gpu, prec, tol):
    import torch

    hm = HMatrix.generate(6000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=3)
    opts, entries = autotune(hm, prec, reps=3)
    # 2 tile shapes x (8 stream + 8 tile-kernel configs) for plain plans, 2 x 8 for mixed, plus combinations
    assert len(entries) >= (32 if prec == "fp64" else 16)
    best = [e for e in entries if e["best"]]
    assert len(best) == 1
    assert best[0]["total_ms"] == min(e["total_ms"] for e in entries)
    assert opts["stage1_cfg"] == best[0]["stage1_cfg"] and opts["stage2_cfg"] == best[0]["stage2_cfg"]
    x = np.random.default_rng(0).uniform(-1, 1, hm.nd)
    with Plan(hm, prec, **opts) as plan:
        info = plan.info()
        assert (info["stage1_cfg"], info["stage2_cfg"]) == (opts["stage1_cfg"], opts["stage2_cfg"])
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        plan.apply(xd, yd)
        torch.cuda.synchronize()
        assert relerr(yd.cpu().numpy(), oracle_hmvm(hm, x)) <= tol


def test_autotune_cache_reuses_a_choice(gpu, tmp_path):
    import torch

    cache = tmp_path / "tune.txt"
    a = HMatrix.generate(6000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=3)
    opts_a, entries_a, hit_a = autotune_cached(a, "fp64", cache, reps=2)
    assert not hit_a and len(entries_a) >= 32 and cache.read_text().count("hmvm_tune 1 ") == 1
    # a smaller matrix of the same family: the stored choice, no sweep
    b = HMatrix.generate(5000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=9)
    opts_b, entries_b, hit_b = autotune_cached(b, "fp64", cache, reps=2)
    assert hit_b and opts_b == opts_a and len(entries_b) == 1
    x = np.random.default_rng(2).uniform(-1, 1, b.nd)
    with Plan(b, "fp64", **opts_b) as plan:
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        plan.apply(xd, yd)
        torch.cuda.synchronize()
        assert relerr(yd.cpu().numpy(), oracle_hmvm(b, x)) <= 1e-12
    # another precision is not the same class: it sweeps and adds its own line
    _, _, hit_m = autotune_cached(b, "mixed", cache, reps=2)
    assert not hit_m and cache.read_text().count("hmvm_tune 1 ") == 2
