"""The reference-signature C++ entry points (include/hmvm_cuda_b200.hpp) used
from a driver shaped like the reference's src_hmvm/src_cpp/hmvm1.cpp."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix
from helpers import REF_INC, ROOT, oracle_hmvm, relerr

DRIVER = os.path.join(ROOT, "tests", "cxx", "hmvm1_b200.cpp")
CUDA = "/usr/local/cuda"


def _compile(out, hacapk_dir):
    lib = os.path.join(ROOT, "hacapk_hmvm_b200")
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", f"-I{hacapk_dir}", f"-I{ROOT}/include",
           f"-I{CUDA}/include", DRIVER, "-o", out, f"-L{lib}", "-lhmvm_b200", f"-L{CUDA}/lib64", "-lcudart",
           f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{CUDA}/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_driver_compiles_against_both_headers(tmp_path):
    _compile(str(tmp_path / "drv_ours"), os.path.join(ROOT, "include"))
    if os.path.exists(os.path.join(REF_INC, "hacapk.h")):
        # the layout static_asserts in the shim check the reference's own templates
        _compile(str(tmp_path / "drv_ref"), REF_INC)


@pytest.mark.gpu
def test_driver_runs(gpu, tmp_path):
    exe = str(tmp_path / "drv")
    _compile(exe, os.path.join(ROOT, "include"))
    hm = HMatrix.generate(2500, "cube", eps=1e-4, seed=9)
    fn = str(tmp_path / "hmatrix_1.bin")
    hm.write_bin1(fn)
    r = subprocess.run([exe, fn, "1", "3"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("TIME")]
    assert len(lines) == 2 and "hmvm_cuda2_b200_k0_d" in lines[0] and "hmvm_cuda2_b200_k0_f" in lines[1]
    x = np.sin(np.arange(1, hm.nd + 1, dtype=np.float64))
    y = np.fromfile(tmp_path / "result_raw_d.bin", dtype=np.float64)
    yo = oracle_hmvm(hm, x)
    assert relerr(y, yo) <= 1e-12
    dump = np.loadtxt(tmp_path / "result_cuda2_b200_k0_d.txt")
    assert np.allclose(dump, yo, rtol=1e-3, atol=1e-3 * np.abs(yo).max())
    dumpf = np.loadtxt(tmp_path / "result_cuda2_b200_k0_f.txt")
    assert relerr(dumpf, yo) <= 1e-3  # %.3E text of the FP32 result
