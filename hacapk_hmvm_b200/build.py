"""In-tree build of the native libraries.

    libhmvm_b200.so  the HMVM library: host planner + sm_100a kernels + C ABI
                     (nvcc -gencode arch=compute_100a,code=sm_100a)
    libhmvm_b200_checked.so
                     the same built with HMVM_DEVICE_CHECKS: descriptor bounds
                     checks on the device before every single-vector stage
                     (loaded instead when HMVM_B200_DEVICE_CHECKS=1)
    libhgen.so       the H-matrix generator / writer (host C++, OpenMP)

Run ``python -m hacapk_hmvm_b200.build`` (or ``__graft_entry__.build()``).  The
built files sit next to this module so they travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

LIB_HMVM = os.path.join(PKG, "libhmvm_b200.so")
LIB_HMVM_CHECKED = os.path.join(PKG, "libhmvm_b200_checked.so")
LIB_HGEN = os.path.join(PKG, "libhgen.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _hostcxx() -> str:
    # The image's CC/CXX wrappers lack the OpenMP spec files; use the system compiler.
    for c in ("/usr/bin/g++", shutil.which("g++") or "g++"):
        if os.path.exists(c):
            return c
    return "g++"


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def hmvm_sources() -> list[str]:
    return [os.path.join(CSRC, f) for f in ("hmvm_b200.cu", "layout.cpp", "layout_tc.cpp", "loader.cpp", "tune.cpp", "solve.cu", "aca.cu")]


def hmvm_deps() -> list[str]:
    deps = hmvm_sources() + [os.path.join(CSRC, f) for f in ("kernels.cuh", "kernels_multi.cuh", "kernels_tc.cuh", "kernels_tcw.cuh", "layout.hpp", "numfmt.hpp", "validate.hpp")]
    deps += [os.path.join(INCLUDE, "hmvm_b200.h"), os.path.join(INCLUDE, "hacapk_hgen.h")]
    return deps


def build_hmvm(force: bool = False, verbose: bool = False, extra: list[str] | None = None,
               checked: bool = False) -> str:
    out = LIB_HMVM_CHECKED if checked else LIB_HMVM
    if not force and not _stale(out, hmvm_deps()):
        return out
    tmp = out + ".tmp"
    cmd = [
        _nvcc(), "-O3", "-std=c++17", "-lineinfo", *ARCH,
        "-ccbin", _hostcxx(),
        "-Xcompiler", "-fPIC,-fopenmp,-O3",
        "-Xptxas", "-warn-spills",
        "-I", INCLUDE, "-I", CSRC,
        "-shared", "-o", tmp, *hmvm_sources(), "-lgomp",
    ]
    if checked:
        cmd[1:1] = ["-DHMVM_DEVICE_CHECKS"]
    if extra:
        cmd[1:1] = extra
    _run(cmd, verbose)
    os.replace(tmp, out)
    return out


def build_hgen(force: bool = False, verbose: bool = False) -> str:
    src = os.path.join(CSRC, "hgen.cpp")
    deps = [src, os.path.join(INCLUDE, "hacapk_hgen.h")]
    if not force and not _stale(LIB_HGEN, deps):
        return LIB_HGEN
    tmp = LIB_HGEN + ".tmp"
    _run([_hostcxx(), "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-Wall",
          "-I", INCLUDE, "-o", tmp, src], verbose)
    os.replace(tmp, LIB_HGEN)
    return LIB_HGEN


def build_all(force: bool = False, verbose: bool = False) -> None:
    from concurrent.futures import ThreadPoolExecutor

    build_hgen(force, verbose)
    with ThreadPoolExecutor(2) as ex:  # the two nvcc runs side by side
        jobs = [ex.submit(build_hmvm, force, verbose, None, c) for c in (False, True)]
        for j in jobs:
            j.result()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
