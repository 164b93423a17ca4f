"""BiCGSTAB on a resident plan (hmvm_b200_bicgstab), the Krylov use of the HMVM
(HACApK_bicgstab_lfmtx, src_lhdump/m_HACApK_solve.f90:977-1028).

* Convergence: the generator's single-layer 1/r matrix is indefinite and
  ill-conditioned (BiCGSTAB stalls on it in exact arithmetic too), so the solve
  runs on H + sigma*I (sigma added to the diagonal of the diagonal dense
  leaves); ||b - H u|| / ||b|| of the returned u, computed in FP64 on the CPU
  with the oracle's HMVM, must be below 10 * eps (FP32: 1e-5, mixed: 2e-4, the
  storage formats' floors).
* Parity: 4 steps on the shifted matrix match a NumPy restatement of the same
  iteration (relative residual and iterate within 1e-7; on the unshifted,
  indefinite matrix the iteration diverges and amplifies rounding differences).
"""
import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, Plan
from helpers import oracle_hmvm

pytestmark = pytest.mark.gpu

_mats = {}


def _mat(shift):
    """The test matrix, with `shift` added to its diagonal."""
    if shift not in _mats:
        hm = HMatrix.generate(3000, "sphere", eta=2.0, eps=1e-6, leaf_size=32, seed=4)
        if shift:
            rm = hm.rowmat.copy()
            for i in range(hm.nlf):
                if hm.ltmtx[i] == 2 and hm.nstrtl[i] == hm.nstrtt[i] and hm.ndl[i] == hm.ndt[i]:
                    n = int(hm.ndt[i])
                    rm[int(hm.a1[i]) + np.arange(n) * (n + 1)] += shift
            hm = HMatrix.from_arrays(hm.nd, hm.ktmax, hm.ltmtx, hm.kt, hm.ndl, hm.ndt, hm.nstrtl, hm.nstrtt, hm.a1,
                                     hm.a2, rm)
        _mats[shift] = hm
    return _mats[shift]


def _numpy_bicgstab(A_mv, b, steps):
    u = np.zeros_like(b)
    r = b - A_mv(u)
    sh, p, akp = r.copy(), np.zeros_like(b), np.zeros_like(b)
    beta = zeta = 0.0
    for _ in range(steps):
        p = r + beta * (p - zeta * akp)
        akp = A_mv(p)
        nom = sh @ r
        alpha = nom / (sh @ akp)
        t = r - alpha * akp
        akt = A_mv(t)
        zeta = (akt @ t) / (akt @ akt)
        u = u + alpha * p + zeta * t
        r = t - zeta * akt
        beta = alpha / zeta * (sh @ r) / nom
    return u, np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("prec,eps,check", [("fp64", 1e-10, 1e-9), ("mixed", 1e-8, 2e-4), ("fp32", 1e-5, 1e-4)])
def test_bicgstab_converges(gpu, prec, eps, check):
    import torch

    hm = _mat(300.0)
    u_true = np.random.default_rng(3).uniform(-1, 1, hm.nd)
    b = oracle_hmvm(hm, u_true)
    dt = torch.float32 if prec == "fp32" else torch.float64
    with Plan(hm, prec) as plan:
        bd = torch.from_numpy(b).to("cuda", dt)
        ud = torch.zeros_like(bd)
        steps, rel = plan.bicgstab(bd, ud, eps=eps, max_steps=200)
        assert 0 < steps < 200 and rel < eps, (steps, rel)
        ud2 = torch.zeros_like(bd)  # repeatable bit for bit
        assert plan.bicgstab(bd, ud2, eps=eps, max_steps=200) == (steps, rel)
        assert torch.equal(ud, ud2)
        u = ud.cpu().numpy().astype(np.float64)
    res = np.linalg.norm(b - oracle_hmvm(hm, u)) / np.linalg.norm(b)
    assert res < check, res


def test_bicgstab_matches_numpy_iteration(gpu):
    import torch

    hm = _mat(300.0)
    b = np.random.default_rng(5).uniform(-1, 1, hm.nd)
    u_np, rel_np = _numpy_bicgstab(lambda v: oracle_hmvm(hm, v), b, 4)
    with Plan(hm, "fp64") as plan:
        bd = torch.from_numpy(b).cuda()
        ud = torch.zeros_like(bd)
        steps, rel = plan.bicgstab(bd, ud, eps=0.0, max_steps=4)
    assert steps == 4
    assert abs(rel - rel_np) <= 1e-7 * rel_np
    u = ud.cpu().numpy()
    assert np.linalg.norm(u - u_np) <= 1e-7 * np.linalg.norm(u_np)


# ---- GCR(m) -------------------------------------------------------------------

def _numpy_gcrm(A_mv, b, steps, m):
    """HACApK_gcrm_lfmtx (src_lhdump/m_HACApK_solve.f90:1277-1342), 0-based,
    u0 = 0, exactly `steps` steps."""
    u = np.zeros_like(b)
    bnorm = np.linalg.norm(b)
    zr = b - A_mv(u)
    zp, zap, capap = [None] * m, [None] * m, [0.0] * m
    zp[0] = zr.copy()
    zap[0] = A_mv(zp[0])
    for it in range(1, steps + 1):
        ik = (it - 1) % m
        zq = zap[ik]
        znom = zq @ zr
        capap[ik] = zq @ zq
        alpha = znom / capap[ik]
        u = u + alpha * zp[ik]
        zr = zr - alpha * zq
        if it == steps:
            break
        zar = A_mv(zr)
        ikn = it % m
        zp[ikn], zap[ikn] = zr.copy(), zar.copy()
        for il in range(ik + 1):  # at a restart il == ikn is the slot being rebuilt
            zq = zap[il]
            beta = -(zq @ zar) / capap[il]
            zp[ikn] = zp[ikn] + beta * zp[il]
            zap[ikn] = zap[ikn] + beta * zq
    return u, np.linalg.norm(zr) / bnorm


@pytest.mark.parametrize("prec,eps,check", [("fp64", 1e-10, 1e-9), ("mixed", 1e-8, 2e-4), ("fp32", 1e-5, 1e-4)])
def test_gcrm_converges(gpu, prec, eps, check):
    import torch

    hm = _mat(300.0)
    u_true = np.random.default_rng(3).uniform(-1, 1, hm.nd)
    b = oracle_hmvm(hm, u_true)
    dt = torch.float32 if prec == "fp32" else torch.float64
    with Plan(hm, prec) as plan:
        bd = torch.from_numpy(b).to("cuda", dt)
        ud = torch.zeros_like(bd)
        steps, rel = plan.gcrm(bd, ud, eps=eps, max_steps=200, restart=4)
        assert 4 < steps < 200 and rel < eps, (steps, rel)  # restarted at least once
        ud2 = torch.zeros_like(bd)  # repeatable bit for bit
        assert plan.gcrm(bd, ud2, eps=eps, max_steps=200, restart=4) == (steps, rel)
        assert torch.equal(ud, ud2)
        u = ud.cpu().numpy().astype(np.float64)
    res = np.linalg.norm(b - oracle_hmvm(hm, u)) / np.linalg.norm(b)
    assert res < check, res


@pytest.mark.parametrize("m,steps", [(3, 7), (20, 5)])
def test_gcrm_matches_numpy_iteration(gpu, m, steps):
    import torch

    hm = _mat(300.0)
    b = np.random.default_rng(5).uniform(-1, 1, hm.nd)
    u_np, rel_np = _numpy_gcrm(lambda v: oracle_hmvm(hm, v), b, steps, m)
    with Plan(hm, "fp64") as plan:
        bd = torch.from_numpy(b).cuda()
        ud = torch.zeros_like(bd)
        got_steps, rel = plan.gcrm(bd, ud, eps=0.0, max_steps=steps, restart=m)
    assert got_steps == steps
    assert abs(rel - rel_np) <= 1e-7 * rel_np
    u = ud.cpu().numpy()
    assert np.linalg.norm(u - u_np) <= 1e-7 * np.linalg.norm(u_np)


def test_gcrm_rejects_bad_restart(gpu):
    import torch

    hm = _mat(300.0)
    with Plan(hm, "fp64") as plan:
        bd = torch.ones(hm.nd, dtype=torch.float64, device="cuda")
        for m in (0, 65):
            with pytest.raises(RuntimeError):
                plan.gcrm(bd, torch.zeros_like(bd), restart=m)
