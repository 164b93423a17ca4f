"""Writes the golden fixtures under tests/golden/ from the reference's own code.

The reference ships no result vectors, so the golden y vectors are produced by
running the reference's hmvm_seq_2<double,0> / <double,1> / <float,0>
(src_hmvm/src_cpp/hmvm_seq.cpp:154-227, built from its sources into
oracle/_ref by oracle/Makefile) on:

  * small H-matrices generated with HACApK's rules (hgen), stored here as
    hmatrix_1.bin files so the inputs are fixed bytes;
  * a hand-built known-answer matrix with integer entries (exact y);
  * the reference's shipped src_hdump/hmatrix_sample.bin, read in place (only
    its SHA-256, statistics and the golden y are stored here, not the file).

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from hacapk_hmvm_b200 import HMatrix  # noqa: E402
from helpers import SAMPLE_BIN, RefMatrix, ref_available, ref_lib  # noqa: E402

MATRICES = [
    # name, n, geometry, eta, eps, leaf, seed
    ("sphere256", 256, "sphere", 2.0, 1e-4, 16, 101),
    ("cube300", 300, "cube", 1.0, 1e-6, 16, 102),
    ("plate200", 200, "plate", 2.0, 1e-3, 8, 103),
]


def xs(n):
    return {
        "sin": np.sin(np.arange(1, n + 1, dtype=np.float64)),  # hmvm1.cpp:37-41
        "uniform": np.random.default_rng(7).uniform(-1.0, 1.0, n),
    }


def kat_matrix():
    """6x6 leaf list with a rank-2 leaf, a rank-0 leaf and dense leaves of
    small integers (exact arithmetic)."""
    D1 = np.arange(1, 10, dtype=np.float64)
    V = np.array([1, 0, 2, 0, 1, 1], dtype=np.float64)   # [kt=2][ndt=3]
    U = np.array([1, 2, 3, 1, -1, 0], dtype=np.float64)  # [kt=2][ndl=3]
    leaves = [  # ltmtx, ndl, ndt, nstrtl, nstrtt, kt, data
        (2, 3, 3, 1, 1, 0, D1),
        (1, 3, 3, 1, 4, 2, np.concatenate([V, U])),
        (1, 3, 3, 4, 1, 0, np.zeros(0)),
        (2, 2, 2, 4, 4, 0, np.array([2.0, 0, 0, 3])),
        (2, 2, 1, 4, 6, 0, np.array([1.0, -1.0])),
        (2, 1, 2, 6, 4, 0, np.array([5.0, 7.0])),
        (2, 1, 1, 6, 6, 0, np.array([-4.0])),
    ]
    a1, a2, off = [], [], 0
    for lt, ndl, ndt, sl, st, kt, d in leaves:
        a1.append(off)
        a2.append(off + kt * ndt if lt == 1 else 0)
        off += d.size
    return HMatrix.from_arrays(6, 2, [l[0] for l in leaves], [l[5] for l in leaves], [l[1] for l in leaves],
                               [l[2] for l in leaves], [l[3] for l in leaves], [l[4] for l in leaves], a1, a2,
                               np.concatenate([l[6] for l in leaves]))


def main():
    if not ref_available():
        sys.exit("oracle/_ref/libhmvm_ref.so is missing: run `make -C oracle` where the reference is present")
    meta = {"matrices": {}, "sample": None}
    out = {}
    for name, n, geo, eta, eps, leaf, seed in MATRICES + [("kat6", None, None, None, None, None, None)]:
        if name == "kat6":
            hm = kat_matrix()
        else:
            hm = HMatrix.generate(n, geo, eta=eta, eps=eps, leaf_size=leaf, seed=seed)
        path = os.path.join(HERE, f"{name}_hmatrix_1.bin")
        hm.write_bin1(path)
        ref = RefMatrix(HMatrix.load(path, 1))
        for xname, x in xs(hm.nd).items():
            out[f"{name}/x_{xname}"] = x
            out[f"{name}/y_seq2_d_{xname}"] = ref.seq2(x, 0)
            out[f"{name}/y_seq2i_d_{xname}"] = ref.seq2(x, 1)
            out[f"{name}/y_seq2_f_{xname}"] = ref.seq2_f(x.astype(np.float32), 0)
        ref.close()
        meta["matrices"][name] = {
            "file": os.path.basename(path), "nd": hm.nd, "nlf": hm.nlf, "ktmax": hm.ktmax, "len": hm.len,
            "sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
            "params": None if name == "kat6" else dict(n=n, geometry=geo, eta=eta, eps=eps, leaf=leaf, seed=seed),
        }
    if os.path.exists(SAMPLE_BIN):
        lib = ref_lib()
        h = lib.ref_load1(SAMPLE_BIN.encode())
        info = np.zeros(4, np.int32)
        lib.ref_info(h, info.ctypes.data)
        nd = int(info[0])
        x = np.sin(np.arange(1, nd + 1, dtype=np.float64))
        y = np.empty(nd)
        lib.ref_seq2_d(h, x.ctypes.data, y.ctypes.data, 0)
        out["sample/y_seq2_d_sin"] = y.copy()
        lib.ref_seq1_d(h, x.ctypes.data, y.ctypes.data, 0)
        out["sample/y_seq1_d_sin"] = y.copy()
        lib.ref_make_float(h)
        xf = np.sin(np.arange(1, nd + 1, dtype=np.float32))  # hmvm1.cpp:112-114 (sin of a float)
        yf = np.empty(nd, np.float32)
        lib.ref_seq2_f(h, xf.ctypes.data, yf.ctypes.data, 0)
        out["sample/y_seq2_f_sin"] = yf
        lib.ref_free(h)
        meta["sample"] = {"nd": nd, "nlf": int(info[1]), "ktmax": int(info[2]), "len": int(info[3]),
                          "sha256": hashlib.sha256(open(SAMPLE_BIN, "rb").read()).hexdigest()}
    np.savez_compressed(os.path.join(HERE, "golden_y.npz"), **out)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(out), "arrays;", ", ".join(meta["matrices"]))


if __name__ == "__main__":
    main()
