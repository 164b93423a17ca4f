"""Leaf fill on the GPU (hmvm_b200_aca_fill): ACA for the low-rank leaves
(HACApK_aca, src_hdump/m_HACApK_base.f90:494-577) and kernel entries for the
dense ones (HACApK_fill_leafmtx_hyp, :580-662) give the same leaf data as the
host generator (hgen_fill_leaves) bit for bit: ranks, offsets and every
element, including leaves that need more than the first capacity round (32
terms) and leaves stopped by kmax."""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from helpers import oracle_hmvm

pytestmark = pytest.mark.gpu

CASES = [
    dict(n=3000, geometry="sphere"),
    dict(n=2500, geometry="cube", leaf_size=20, eta=1.0, eps=1e-6),
    dict(n=2000, geometry="plate", leaf_size=24, eps=1e-10),  # ranks above 32: a second round
    dict(n=2000, geometry="sphere", eps=1e-8, kmax=5),        # every big leaf stopped by kmax
    dict(n=700, geometry="cube", leaf_size=8, eta=0.5, seed=3),
]


def _same(a: HMatrix, b: HMatrix):
    assert (a.nd, a.nlf, a.ktmax, a.len) == (b.nd, b.nlf, b.ktmax, b.len)
    for f in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert np.array_equal(a.rowmat.view(np.uint64), b.rowmat.view(np.uint64))
    assert a.meta["aca_incomplete"] == b.meta["aca_incomplete"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_gpu_fill_bit_identical(gpu, case):
    cpu = HMatrix.generate(**case, fill="cpu")
    dev = HMatrix.generate(**case, fill="gpu")
    _same(cpu, dev)
    rep = dev.meta["aca_report"]
    assert rep["ktmax"] == dev.ktmax and rep["rounds"] >= 1
    if case.get("eps") == 1e-10:
        assert dev.ktmax > 32 and rep["rounds"] >= 2
    if case.get("kmax") == 5:
        assert dev.ktmax == 5 and dev.meta["aca_incomplete"] > 0


def test_gpu_filled_matrix_multiplies(gpu):
    hm = HMatrix.generate(4000, "sphere", seed=7, fill="gpu")
    x = np.random.default_rng(1).uniform(-1, 1, hm.nd)
    with Plan(hm, "fp64") as plan:
        y = plan.apply_host(x)
    yo = oracle_hmvm(hm, x)
    assert np.linalg.norm(y - yo) <= 1e-12 * np.linalg.norm(yo)
