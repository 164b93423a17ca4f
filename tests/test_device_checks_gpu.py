"""The HMVM_DEVICE_CHECKS build (hacapk_hmvm_b200/libhmvm_b200_checked.so,
loaded when HMVM_B200_DEVICE_CHECKS=1): before every single-vector stage it
checks the stage's descriptors on the device (csrc/validate.hpp).  On valid
plans it reports no error, launches one validation per stage, and gives the
same y bit for bit as the normal build.  Each build runs in its own process,
since the environment variable picks the library at load time."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = [
    (2048, "sphere", "fp64", {}),
    (2048, "sphere", "fp32", {}),
    (2048, "sphere", "mixed", {}),
    (1500, "cube", "fp64", {"kernel": 0}),
    (3000, "plate", "mixed", {"split_cols": 8}),
    (1201, "cube", "fp32", {"max_tile_rows": 7}),
]
SCRIPT = r"""
import hashlib, json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from hacapk_hmvm_b200 import HMatrix, Plan, _lib
out = {"lib": _lib.LIB_HMVM_PATH, "runs": []}
for n, geo, prec, opts in json.loads(sys.argv[2]):
    hm = HMatrix.generate(n, geo, eta=2.0, eps=1e-4, leaf_size=32, seed=7)
    x = np.random.default_rng(3).uniform(-1, 1, hm.nd)
    with Plan(hm, prec, **opts) as plan:
        dt = torch.float32 if prec == "fp32" else torch.float64
        xd = torch.from_numpy(x).to("cuda", dt)
        yd = torch.full_like(xd, float("nan"))
        for _ in range(2):
            plan.apply(xd, yd)
        torch.cuda.synchronize()
        plan.status()
        y = yd.cpu().numpy()
        out["runs"].append({"kernels": plan.kernel_count(), "v_stage": plan.info()["stage1_tiles"] > 0,
                            "finite": bool(np.isfinite(y).all()), "md5": hashlib.md5(y.tobytes()).hexdigest()})
print(json.dumps(out))
"""


def _run(checked: bool) -> dict:
    env = dict(os.environ, HMVM_B200_DEVICE_CHECKS="1" if checked else "0")
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, json.dumps(CASES)], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_matches_the_normal_build(gpu):
    from hacapk_hmvm_b200 import build

    if not os.path.exists(build.LIB_HMVM_CHECKED):
        pytest.fail("libhmvm_b200_checked.so is missing: build() builds it")
    plain, checked = _run(False), _run(True)
    assert plain["lib"].endswith("libhmvm_b200.so")
    assert checked["lib"].endswith("libhmvm_b200_checked.so")
    for case, a, b in zip(CASES, plain["runs"], checked["runs"]):
        assert a["finite"] and b["finite"], case
        assert a["md5"] == b["md5"], case  # same kernels, same order: bit for bit
        assert b["kernels"] == a["kernels"] + (2 if a["v_stage"] else 1), case  # one validation per stage


NEG_SCRIPT = r"""
import ctypes as C, json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from hacapk_hmvm_b200 import HMatrix, Plan, _lib
lib = _lib.hmvm_lib()
hm = HMatrix.generate(2048, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=7)
x = np.random.default_rng(3).uniform(-1, 1, hm.nd)
res = {"lib": _lib.LIB_HMVM_PATH}
with Plan(hm, "fp64") as plan:
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    plan.apply(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    y0 = yd.cpu().numpy().copy()
    ptr, n, n1 = C.c_void_p(), C.c_int32(), C.c_int32()
    _lib.check(lib.hmvm_b200_plan_descriptors(plan.handle, C.byref(ptr), C.byref(n), C.byref(n1)), "descriptors")

    class Mem:
        pass

    mem = Mem()
    mem.__cuda_array_interface__ = {"shape": (n.value * 32,), "typestr": "|u1", "data": (ptr.value, False),
                                    "version": 3}
    # hmvm_tile_desc as 8 int32: data_off (2), seg_begin, nseg, nvec, out_base, nrows | mode, _pad
    tiles = torch.as_tensor(mem, device="cuda").view(torch.int32).view(n.value, 8)
    k = next(k for k in range(n1.value, n.value) if tiles[k, 4].item() >= 2)
    tiles[k, 4] -= 1  # one vector fewer than its segments hold: flagged, and in bounds even if followed
    torch.cuda.synchronize()
    plan.apply(xd, yd)
    torch.cuda.synchronize()
    try:
        plan.status()
        res["caught"] = False
    except _lib.HMVMError as e:
        res["caught"] = e.status == _lib.HMVM_EDEVICE
        res["msg"] = str(e)
    tiles[k, 4] += 1
    torch.cuda.synchronize()
    plan.apply(xd, yd)
    torch.cuda.synchronize()
    plan.status()
    res["restored"] = bool(np.array_equal(yd.cpu().numpy().view(np.uint64), y0.view(np.uint64)))
print(json.dumps(res))
"""


def test_checked_build_reports_a_changed_descriptor(gpu):
    """A row item's vector count changed on the device after the plan was
    made: the checked build's validation reports it (HMVM_EDEVICE, device
    bounds check) and the row stage touches nothing; restored, the same plan
    gives the original y bit for bit."""
    env = dict(os.environ, HMVM_B200_DEVICE_CHECKS="1")
    r = subprocess.run([sys.executable, "-c", NEG_SCRIPT, ROOT], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["lib"].endswith("libhmvm_b200_checked.so")
    assert res["caught"], res
    assert "device bounds check" in res["msg"], res
    assert res["restored"], res
