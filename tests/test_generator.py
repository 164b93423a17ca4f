"""The H-matrix generator (include/hacapk_hgen.h): HACApK's construction rules
hold on its output, the reference's own loaders read its files, and from the
reference's sample mesh it rebuilds the reference's sample matrix."""
import os

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix
from helpers import SAMPLE_BIN, SAMPLE_PBF, RefMatrix, ref_available, relerr


def _boxes(hm, r0, n):
    pts = hm.meta["coords"][hm.meta["lod"][r0:r0 + n] - 1]
    return pts.min(axis=0), pts.max(axis=0)


@pytest.mark.parametrize("geo,eta,eps,leaf", [("sphere", 2.0, 1e-4, 32), ("cube", 1.0, 1e-6, 16),
                                              ("plate", 2.0, 1e-3, 8)])
def test_structure(geo, eta, eps, leaf):
    hm = HMatrix.generate(1500, geo, eta=eta, eps=eps, leaf_size=leaf, seed=4)
    n = hm.nd
    # leaves tile the n x n matrix exactly once
    cov = np.zeros((n, n), np.int8)
    for i in range(hm.nlf):
        r, c = hm.nstrtl[i] - 1, hm.nstrtt[i] - 1
        cov[r:r + hm.ndl[i], c:c + hm.ndt[i]] += 1
    assert np.all(cov == 1)
    # rows nondecreasing (HACApK's row sort, m_HACApK_base.f90:245)
    assert np.all(np.diff(hm.nstrtl) >= 0)
    # lod is a permutation
    assert np.array_equal(np.sort(hm.meta["lod"]), np.arange(1, n + 1))
    lr = hm.ltmtx == 1
    # admissibility of every low-rank leaf and size rules (:860-877)
    for i in np.where(lr)[0]:
        lo1, hi1 = _boxes(hm, hm.nstrtl[i] - 1, hm.ndl[i])
        lo2, hi2 = _boxes(hm, hm.nstrtt[i] - 1, hm.ndt[i])
        gap = np.maximum(0, np.maximum(lo2 - hi1, lo1 - hi2))
        dist = np.sqrt((gap ** 2).sum())
        w1, w2 = np.linalg.norm(hi1 - lo1), np.linalg.norm(hi2 - lo2)
        assert min(w1, w2) <= eta * dist * (1 + 1e-12)
        assert hm.ndl[i] >= leaf + 1 and hm.ndt[i] >= leaf + 1
    assert hm.ktmax == hm.kt[lr].max()
    assert hm.meta["aca_incomplete"] == 0


def test_aca_accuracy_and_entries():
    hm = HMatrix.generate(2000, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=6)
    rm = hm.rowmat
    errs = []
    for i in np.where(hm.ltmtx == 1)[0][:40]:
        k, l, t = hm.kt[i], hm.ndl[i], hm.ndt[i]
        V = rm[hm.a1[i]:hm.a1[i] + k * t].reshape(k, t)
        U = rm[hm.a2[i]:hm.a2[i] + k * l].reshape(k, l)
        E = np.array([[hm.entry(hm.nstrtl[i] + r, hm.nstrtt[i] + c) for c in range(t)] for r in range(l)])
        errs.append(np.linalg.norm(U.T @ V - E) / np.linalg.norm(E))
    assert max(errs) < 1e-2 and np.median(errs) < 1e-3
    # dense leaves hold exact kernel entries; the diagonal is the self term 1.0
    for i in np.where(hm.ltmtx == 2)[0][:20]:
        l, t = hm.ndl[i], hm.ndt[i]
        D = rm[hm.a1[i]:hm.a1[i] + l * t].reshape(l, t)
        E = np.array([[hm.entry(hm.nstrtl[i] + r, hm.nstrtt[i] + c) for c in range(t)] for r in range(l)])
        assert np.array_equal(D, E)
    assert hm.entry(5, 5) == 1.0


def test_deterministic():
    a = HMatrix.generate(3000, "cube", seed=12, nthreads=1)
    b = HMatrix.generate(3000, "cube", seed=12, nthreads=4)
    assert np.array_equal(a.rowmat, b.rowmat) and np.array_equal(a.kt, b.kt)
    c = HMatrix.generate(3000, "cube", seed=13)
    assert not np.array_equal(a.rowmat[:100], c.rowmat[:100])


@pytest.mark.skipif(not ref_available(), reason="reference build oracle/_ref absent")
def test_reference_reads_generated_files(tmp_path):
    import ctypes as C

    from helpers import ref_lib

    hm = HMatrix.generate(1000, "sphere", seed=2)
    p1, p2 = str(tmp_path / "hmatrix_1.bin"), str(tmp_path / "hmatrix_2.bin")
    hm.write_bin1(p1)
    hm.write_bin2(p2)
    r = ref_lib()
    x = np.sin(np.arange(1, hm.nd + 1, dtype=np.float64))
    h1, h2 = r.ref_load1(p1.encode()), r.ref_load2(p2.encode())
    y1, y2, y3 = np.empty(hm.nd), np.empty(hm.nd), np.empty(hm.nd)
    r.ref_seq1_d(h1, x.ctypes.data, y1.ctypes.data, 0)  # AoS from hmatrix_1.bin
    r.ref_seq2_d(h1, x.ctypes.data, y2.ctypes.data, 0)  # SoA from hmatrix_1.bin
    r.ref_seq2_d(h2, x.ctypes.data, y3.ctypes.data, 0)  # SoA from hmatrix_2.bin
    r.ref_free(h1)
    r.ref_free(h2)
    assert np.array_equal(y1, y2) and np.array_equal(y2, y3)
    # and it approximates the dense kernel matrix to the ACA tolerance
    A = np.array([[hm.entry(i, j) for j in range(1, hm.nd + 1)] for i in range(1, hm.nd + 1)])
    assert relerr(y2, A @ x) < 1e-3


def test_write_rejects_range(tmp_path):
    # a leaf record beyond the format's int32 byte count is refused, not wrapped
    hm = HMatrix.from_arrays(1, 1, [2], [0], [1], [1], [1], [1], [0], [0], np.array([1.0]))
    hm.write_bin1(str(tmp_path / "ok.bin"))
    assert HMatrix.load(str(tmp_path / "ok.bin")).rowmat[0] == 1.0


def test_tree_then_fill_equals_build():
    """hgen_build == hgen_build_tree + hgen_fill_leaves, and the tree alone
    carries no leaf data."""
    import ctypes as C

    from hacapk_hmvm_b200 import _lib

    lib = _lib.hgen_lib()
    p = _lib.HgenParams()
    lib.hgen_default_params(C.byref(p))
    p.n, p.geometry, p.eps, p.seed = 1500, 1, 1e-5, 11
    whole, tree = C.POINTER(_lib.HgenMatrix)(), C.POINTER(_lib.HgenMatrix)()
    assert lib.hgen_build(C.byref(p), C.byref(whole)) == 0
    assert lib.hgen_build_tree(C.byref(p), C.byref(tree)) == 0
    try:
        t = tree.contents
        assert not t.rowmat and t.len == 0 and t.nlf == whole.contents.nlf
        assert lib.hgen_fill_leaves(tree, C.byref(p)) == 0
        assert lib.hgen_fill_leaves(tree, C.byref(p)) != 0  # already filled
        w = whole.contents
        assert (t.len, t.ktmax, t.aca_incomplete) == (w.len, w.ktmax, w.aca_incomplete)
        n = w.nlf
        for f in ("ltmtx", "kt", "ndl", "ndt", "nstrtl", "nstrtt", "a1", "a2"):
            dt = np.int64 if f in ("a1", "a2") else np.int32
            assert np.array_equal(np.ctypeslib.as_array(getattr(t, f), (n,)).view(dt),
                                  np.ctypeslib.as_array(getattr(w, f), (n,)).view(dt)), f
        assert np.array_equal(np.ctypeslib.as_array(t.rowmat, (t.len,)), np.ctypeslib.as_array(w.rowmat, (w.len,)))
    finally:
        lib.hgen_free(whole)
        lib.hgen_free(tree)


def test_gpu_fill_refuses_without_device():
    """hmvm_b200_aca_fill returns a status (no crash) where no sm_100 device is
    usable, and leaves the matrix unfilled."""
    import ctypes as C

    import torch

    from hacapk_hmvm_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.hgen_lib()
    p = _lib.HgenParams()
    lib.hgen_default_params(C.byref(p))
    p.n = 600
    tree = C.POINTER(_lib.HgenMatrix)()
    assert lib.hgen_build_tree(C.byref(p), C.byref(tree)) == 0
    try:
        rep = _lib.AcaReport()
        rc = _lib.hmvm_lib().hmvm_b200_aca_fill(tree, C.byref(p), 0, C.byref(rep))
        assert rc == _lib.HMVM_ENODEV and not tree.contents.rowmat
    finally:
        lib.hgen_free(tree)


# ---- ppohBEM meshes: the reference's own sample matrix --------------------------


@pytest.mark.skipif(not (os.path.exists(SAMPLE_PBF) and os.path.exists(SAMPLE_BIN)),
                    reason="the reference's sample mesh and matrix are not present")
def test_mesh_reproduces_reference_sample():
    """HACApK built src_hdump/hmatrix_sample.bin from input_sample.pbf with the
    ppohBEM collocation kernel (leaf 15, eta 2, tolerance 1e-6 from
    bem-bb-config.txt).  The generator, given the same mesh, rebuilds the same
    leaf list -- every leaf's position, size, type and ACA rank -- and the same
    values up to the last bits of libm's atan2/log (dense entries within 1e-12
    relative; the HMVM within 1e-13)."""
    ref = HMatrix.load(SAMPLE_BIN)
    ours = HMatrix.from_mesh(SAMPLE_PBF)
    assert (ours.nd, ours.nlf, ours.ktmax, ours.len) == (ref.nd, ref.nlf, ref.ktmax, ref.len) == (600, 1426, 31, 248662)
    for f in ("ltmtx", "ndl", "ndt", "nstrtl", "nstrtt", "kt", "a1", "a2"):
        assert np.array_equal(getattr(ours, f), getattr(ref, f)), f
    dense = np.nonzero(ref.ltmtx == 2)[0]
    for i in dense:
        n = int(ref.ndl[i]) * int(ref.ndt[i])
        a, b = ref.rowmat[ref.a1[i]:ref.a1[i] + n], ours.rowmat[ours.a1[i]:ours.a1[i] + n]
        assert np.all(np.abs(a - b) <= 1e-12 * np.abs(a)), i
    x = np.sin(np.arange(1, ref.nd + 1, dtype=np.float64))  # the reference harness's b[i] = sin(i+1)
    from helpers import oracle_hmvm

    y_ref, y = oracle_hmvm(ref, x), oracle_hmvm(ours, x)
    assert relerr(y, y_ref) < 1e-13
    # the entries are the kernel's: a dense leaf's values equal entry(i, j)
    i = int(dense[0])
    r, c = int(ours.nstrtl[i]), int(ours.nstrtt[i])
    assert ours.entry(r, c) == ours.rowmat[ours.a1[i]]


@pytest.mark.parametrize("fault", ["missing", "truncated", "node_index", "not_a_number"])
def test_pbf_reader_faults(tmp_path, fault):
    import ctypes as C

    from hacapk_hmvm_b200 import _lib

    good = "4\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n2\n3\n0\n1\n0 1 2\n0 1 3\n-1.0\n-1.0\n"
    text = {"truncated": good[:40], "node_index": good.replace("0 1 3", "0 1 4"),
            "not_a_number": good.replace("1 0 0", "1 x 0"), "missing": None}[fault]
    p = str(tmp_path / "m.pbf")
    if text is not None:
        open(p, "w").write(text)
    lib = _lib.hgen_lib()
    mesh = C.POINTER(_lib.HgenMesh)()
    assert lib.hgen_read_pbf(p.encode(), C.byref(mesh)) == -3 and not mesh  # HGEN_EIO
    open(p, "w").write(good)
    assert lib.hgen_read_pbf(p.encode(), C.byref(mesh)) == 0
    m = mesh.contents
    assert (m.nond, m.nofc, m.nond_on_face, m.nint_para_fc, m.ndble_para_fc) == (4, 2, 3, 0, 1)
    assert [m.face2node[k] for k in range(6)] == [0, 1, 2, 0, 1, 3] and m.dble_para_fc[1] == -1.0
    lib.hgen_free_mesh(mesh)
