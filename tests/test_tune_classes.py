"""Shape classes of the autotuner's cache (hmvm_b200_shape_histogram64), on the
CPU: the histogram is the fraction of stored elements per (kind, rows, width)
class, matrices of one family lie close together whatever their size, and
other geometries or leaf sizes lie far apart."""
import numpy as np

from hacapk_hmvm_b200 import HMatrix, shape_histogram


def _bucket(v, first):
    b, lim = 0, 1 << first
    while b < 7 and v > lim:
        b, lim = b + 1, lim << 1
    return b


def test_histogram_matches_the_leaf_table():
    hm = HMatrix.generate(3000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=3)
    h = shape_histogram(hm)
    want = np.zeros(128)
    for i in range(hm.nlf):
        lr = hm.ltmtx[i] == 1
        el = hm.kt[i] * (hm.ndl[i] + hm.ndt[i]) if lr else hm.ndl[i] * hm.ndt[i]
        width = hm.kt[i] if lr else hm.ndt[i]
        want[(64 if lr else 0) + 8 * _bucket(hm.ndl[i], 3) + _bucket(width, 1 if lr else 3)] += el
    want /= want.sum()
    assert abs(h.sum() - 1.0) < 1e-5
    assert np.allclose(h, want, atol=1e-6)


def test_families_near_others_far():
    base = shape_histogram(HMatrix.generate(6000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=3))
    same = shape_histogram(HMatrix.generate(5000, "cube", eta=2.0, eps=1e-4, leaf_size=32, seed=9))
    geo = shape_histogram(HMatrix.generate(6000, "sphere", eta=2.0, eps=1e-4, leaf_size=32, seed=3))
    leaf = shape_histogram(HMatrix.generate(6000, "plate", eta=1.0, eps=1e-6, leaf_size=16, seed=3))
    d = lambda a, b: float(np.abs(a - b).sum())  # noqa: E731
    assert d(base, same) <= 0.45  # the cache's default bound joins these
    assert d(base, geo) > 0.45 and d(base, leaf) > 0.45
