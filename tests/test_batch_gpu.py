"""Batches of independent H-matrices (hmvm_b200_batch_*) on the GPU.

Instances of uneven N, geometry, eta and ACA tolerance run as block-diagonal
plans (one per pass width) whose passes all run in the same launches, one per
stage; every instance's Y columns are checked against the FP64
oracle on that instance alone (FP32 <= 1e-5, FP64 <= 1e-12, mixed <= 1e-4
relative error per column).  The CUDA-graph replay must give the same bits as
the direct apply.
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import Batch, HMatrix
from helpers import oracle_hmvm, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5, "mixed": 1e-4}
SPECS = [(700, "sphere", 2.0, 1e-4), (1900, "cube", 1.0, 1e-6), (433, "plate", 2.0, 1e-3),
         (2600, "sphere", 1.0, 1e-4), (64, "cube", 2.0, 1e-4), (1200, "plate", 1.0, 1e-6)]
_mats = []


def _instances():
    if not _mats:
        for i, (n, geo, eta, eps) in enumerate(SPECS):
            _mats.append(HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=32, seed=40 + i))
    return _mats


def _blocks(mats, nrhs, dtype, seed=0):
    import torch

    rng = np.random.default_rng(seed)
    Xh = [rng.uniform(-1, 1, (k, m.nd)) for m, k in zip(mats, nrhs)]
    dt = torch.float32 if dtype == np.float32 else torch.float64
    Xs = [torch.from_numpy(x.astype(dtype)).cuda() for x in Xh]
    Ys = [torch.full((k, m.nd), float("nan"), dtype=dt, device="cuda") for m, k in zip(mats, nrhs)]
    return Xh, Xs, Ys


def _check(mats, Xh, Ys, prec):
    for i, (m, x, y) in enumerate(zip(mats, Xh, Ys)):
        Y = y.cpu().numpy().astype(np.float64)
        for r in range(x.shape[0]):
            e = relerr(Y[r], oracle_hmvm(m, x[r]))
            assert e <= TOL[prec], (i, r, e)


@pytest.mark.parametrize("prec,nrhs_max", [("fp32", 8), ("fp32", 1), ("fp64", 4), ("mixed", 8)])
def test_batch_parity(gpu, prec, nrhs_max):
    import torch

    mats = _instances()
    nrhs = [1, 16, 3, 5, 2, 9]
    Xh, Xs, Ys = _blocks(mats, nrhs, np.float32 if prec == "fp32" else np.float64)
    with Batch(mats, prec, nrhs=[min(k, nrhs_max) for k in nrhs]) as b:
        info = b.info()
        assert info["nd"] == sum(m.nd for m in mats)
        b.apply(Xs, Ys)
        torch.cuda.synchronize()
        b.status()
    _check(mats, Xh, Ys, prec)


def test_batch_graph_replay_matches_apply(gpu):
    import torch

    mats = _instances()
    nrhs = [4, 1, 7, 8, 2, 16]
    Xh, Xs, Ys = _blocks(mats, nrhs, np.float32, seed=3)
    _, _, Y2 = _blocks(mats, nrhs, np.float32, seed=3)
    with Batch(mats, "fp32", nrhs=nrhs) as b:
        assert b.class_count() == 4  # (width, passes): (2, 1), (4, 1), (8, 1), (8, 2)
        b.apply(Xs, Ys)
        # one launch for packing, one per stage and reduction, one for unpacking, over all
        # classes and passes (5 parts here: 16 columns take two 8-wide passes)
        assert b.kernel_count() <= 6
        b.apply(Xs, Ys)
        b.capture(Xs, Y2)
        s = torch.cuda.Stream()
        for _ in range(3):
            b.launch(s)
        s.synchronize()
        b.status()
        assert b.kernel_count() > 0
    for y, y2 in zip(Ys, Y2):
        assert torch.equal(y, y2)
    _check(mats, Xh, Y2, "fp32")


def test_batch_skips_empty_instances(gpu):
    import torch

    mats = _instances()
    nrhs = [2, 0, 1, 0, 3, 1]
    Xh, Xs, Ys = _blocks(mats, [max(k, 1) for k in nrhs], np.float64, seed=9)
    Xs = [x[:k] if k else x[:1] for x, k in zip(Xs, nrhs)]
    Ys_used = [y[:k] if k else y[:1] for y, k in zip(Ys, nrhs)]
    with Batch(mats, "fp64", nrhs_max=2) as b:
        assert b.class_count() == 1
        from hacapk_hmvm_b200 import _lib
        import ctypes as C

        t = list(b._tables(Xs, Ys_used))
        t[4] = (C.c_int32 * len(mats))(*nrhs)
        _lib.check(_lib.hmvm_lib().hmvm_b200_batch_apply(b.handle, *t, 0), "batch apply")
        torch.cuda.synchronize()
        assert b.instance(2) == (mats[2].nd, 0, mats[0].nd + mats[1].nd)
    for i, k in enumerate(nrhs):
        Y = Ys[i].cpu().numpy()
        if k == 0:
            assert np.all(np.isnan(Y))
        else:
            for r in range(k):
                assert relerr(Y[r], oracle_hmvm(mats[i], Xh[i][r])) <= TOL["fp64"]
