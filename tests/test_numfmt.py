"""The planner's encoders for the compact storage formats of mixed-precision
plans (csrc/numfmt.hpp): round to nearest, ties to even, from the double.

Checked against an exact rational restatement of rounding on the format's
grid, against numpy's float16 and, for inputs representable in binary32
(where rounding through binary32 is single rounding), torch's bfloat16 and
float8_e4m3fn conversions."""
import ctypes as C
import os
import subprocess
from fractions import Fraction

import numpy as np
import pytest
import torch

from helpers import E4M3

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hacapk_hmvm_b200", "csrc")


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("numfmt") / "libnumfmt_probe.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", so,
                    os.path.join(HERE, "cxx", "numfmt_probe.cpp")], check=True)
    lib = C.CDLL(so)
    lib.probe_encode.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_long]

    def enc(ty, x):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(x.size, np.uint8 if ty == 3 else np.uint16)
        lib.probe_encode(ty, x.ctypes.data, out.ctypes.data, x.size)
        return out

    return enc


def exact_round(v, ebits, mbits, bias, maxfinite):
    """Nearest value of the format's grid to v (ties to even), by rationals;
    saturating at maxfinite."""
    a = abs(Fraction(v))
    if a == 0:
        return 0.0
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if Fraction(2) ** e > a:
        e -= 1
    e = max(e, 1 - bias)
    q = Fraction(2) ** (e - mbits)
    k, r = divmod(a, q)
    k = int(k)
    if r > q / 2 or (r == q / 2 and k % 2):
        k += 1
    val = min(float(k * q), maxfinite)
    return -val if v < 0 else val


def inputs(seed):
    rng = np.random.default_rng(seed)
    x = np.concatenate([
        rng.uniform(-1, 1, 4000),
        rng.standard_normal(2000) * 10.0 ** rng.uniform(-12, 5, 2000),
        np.ldexp(rng.integers(1, 64, 1000).astype(np.float64) + 0.5, rng.integers(-30, 10, 1000)),  # ties
        [0.0, -0.0, 1.0, -1.0, 448.0, 449.0, 464.0, 1e9, 2.0 ** -9, 2.0 ** -10, 3 * 2.0 ** -11, 65504.0,
         65519.0, 2.0 ** -24, 2.0 ** -25, 1.5 * 2.0 ** -25],
    ])
    return x


def test_fp16_matches_numpy(probe):
    x = inputs(0)
    x = x[np.abs(x) < 65520]
    assert np.array_equal(probe(2, x), x.astype(np.float16).view(np.uint16))


def test_fp16_matches_exact_rounding(probe):
    x = inputs(1)[:3000]
    got = probe(2, x).view(np.float16).astype(np.float64)
    want = np.array([exact_round(v, 5, 10, 15, 65504.0) for v in x])
    assert np.array_equal(got, want)


def test_e4m3_matches_exact_rounding(probe):
    x = inputs(2)
    got = E4M3[probe(3, x)]
    want = np.array([exact_round(v, 4, 3, 7, 448.0) for v in x])
    assert np.array_equal(got, want)


def test_e4m3_matches_torch_on_binary32(probe):
    x = inputs(3).astype(np.float32).astype(np.float64)
    x = x[np.abs(x) <= 448.0]
    want = torch.from_numpy(x.astype(np.float32)).to(torch.float8_e4m3fn).view(torch.uint8).numpy()
    assert np.array_equal(probe(3, x), want)


def test_bf16_matches_exact_rounding_and_torch(probe):
    x = inputs(4)
    got = (probe(4, x).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    want = np.array([exact_round(v, 8, 7, 127, 3.3895313892515355e38) for v in x])
    assert np.array_equal(got, want)
    x32 = x.astype(np.float32).astype(np.float64)
    tb = torch.from_numpy(x32.astype(np.float32)).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(probe(4, x32), tb)


def test_special_values(probe):
    assert probe(2, [np.inf, -np.inf, 1e6]).tolist() == [0x7C00, 0xFC00, 0x7C00]
    assert probe(3, [1e6, -1e6, np.nan]).tolist() == [0x7E, 0xFE, 0x7F]
    assert probe(4, [np.inf, 3.4e38, np.nan]).tolist() == [0x7F80, 0x7F80, 0x7FC0]
