"""The C ABI: every function the public headers declare is exported by the
built libraries, the ctypes mirrors have the headers' layouts, and calls that
need a GPU fail with a status (never a crash or a CPU fallback) without one."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from hacapk_hmvm_b200 import HMatrix, _lib
from helpers import ROOT

INC = os.path.join(ROOT, "include")


def declared(header):
    src = open(os.path.join(INC, header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M))
    return {n for n in names if n.startswith(("hmvm_", "hgen_"))}


def test_every_declared_function_is_exported():
    hm = declared("hmvm_b200.h")
    hg = declared("hacapk_hgen.h")
    assert {"hmvm_b200_apply", "hmvm_b200_apply_noalloc", "hmvm_cuda_d", "hmvm_b200_load_hmatrix"} <= hm
    lib_h, lib_g = C.CDLL(_lib.LIB_HMVM_PATH), C.CDLL(_lib.LIB_HGEN_PATH)
    for n in hm:
        assert hasattr(lib_h, n), n
    for n in hg:
        assert hasattr(lib_g, n), n
    # and the Python binding knows every one of them
    assert hm <= set(_lib.HMVM_SIGNATURES)
    assert hg <= set(_lib.HGEN_SIGNATURES)


STRUCTS = {
    "hmvm_matrix2_d": _lib.Matrix2_d, "hmvm_matrix2_f": _lib.Matrix2_f, "hmvm_matrix_d": _lib.Matrix_d,
    "hmvm_submatrix_d": _lib.Submatrix_d, "hmvm_leaves64": _lib.Leaves64, "hmvm_plan_opts": _lib.PlanOpts,
    "hmvm_plan_info": _lib.PlanInfo, "hmvm_stats": _lib.Stats, "hmvm_tile_desc": _lib.TileDesc,
    "hmvm_seg_desc": _lib.SegDesc, "hmvm_layout_view": _lib.LayoutView, "hmvm_tune_entry": _lib.TuneEntry,
    "hmvm_tune_report": _lib.TuneReport,
}


def test_struct_layouts_match_headers(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hmvm_b200.h"', '#include "hacapk_hgen.h"',
             "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    for cname, py in (("hgen_params", _lib.HgenParams), ("hgen_hmatrix", _lib.HgenMatrix)):
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        STRUCTS[cname] = py
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", INC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        key, val = line.split()
        if "." in key:
            s, f = key.split(".")
            assert getattr(STRUCTS[s], f).offset == int(val), key
        else:
            assert C.sizeof(STRUCTS[key]) == int(val), key


def test_reference_struct_bytes():
    # matrix2<double> of src_hmvm/src_cpp/hacapk.h: 4 ints, 11 pointers, 2 ints, 2 pointers
    assert C.sizeof(_lib.Matrix2_d) == 4 * 4 + 11 * 8 + 2 * 4 + 2 * 8
    assert _lib.Matrix2_d.rowmat.offset == 16 + 9 * 8


def test_status_strings():
    lib = _lib.hmvm_lib()
    for code in range(-8, 1):
        assert lib.hmvm_b200_strerror(code)
    assert lib.hmvm_b200_version() >= 1


def test_layout_api_needs_no_gpu():
    from helpers import layout_for

    hm = HMatrix.generate(500, "sphere", seed=1)
    h, v = layout_for(hm, precision=0)
    assert v.n_tiles > 0 and v.data_vectors > 0
    _lib.hmvm_lib().hmvm_b200_layout_destroy(h)


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a GPU")
def test_no_device_is_an_error_not_a_fallback():
    hm = HMatrix.generate(300, "cube", seed=1)
    lib = _lib.hmvm_lib()
    o = _lib.PlanOpts()
    lib.hmvm_b200_default_opts(C.byref(o))
    h = C.c_void_p()
    m2 = hm.as_matrix2()
    assert lib.hmvm_b200_plan_create_d(C.byref(m2), C.byref(o), C.byref(h)) == _lib.HMVM_ENODEV
    assert not h
    y = np.zeros(hm.nd)
    x = np.ones(hm.nd)
    assert lib.hmvm_cuda_d(C.byref(m2), x.ctypes.data, y.ctypes.data, 0, None) == _lib.HMVM_ENODEV
    assert not y.any()
    assert lib.hmvm_b200_apply(None, None, None, None) == _lib.HMVM_EINVAL
