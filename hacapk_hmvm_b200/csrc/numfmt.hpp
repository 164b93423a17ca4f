// Host-side conversions to the compact storage formats of the mixed-precision
// layout, written from the format definitions (round to nearest, ties to even):
//   IEEE 754 binary16 (1 sign, 5 exponent bits, bias 15, 10 fraction bits),
//   bfloat16 (1 sign, 8 exponent bits, bias 127, 7 fraction bits),
//   OCP FP8 E4M3 "fn" (1 sign, 4 exponent bits, bias 7, 3 fraction bits; no
//   infinities, 0x7f/0xff are NaN, largest finite 448; values beyond are
//   saturated to +-448 here).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace hmvm {

// Round a finite |v| to the grid k * 2^e2 (nearest, ties to even); returns k.
inline uint64_t round_to_grid(double a, int e2) {
  double q = std::ldexp(a, -e2);  // exact: scaling by a power of two
  double f = std::floor(q);
  double r = q - f;
  uint64_t k = (uint64_t)f;
  if (r > 0.5 || (r == 0.5 && (k & 1))) k++;
  return k;
}

// Encode |a| (finite, >= 0) into a format with `ebits` exponent bits, `mbits`
// fraction bits and bias `bias`, largest finite value `maxv`; returns the
// unsigned bit pattern (no sign).  Saturates above maxv.
inline uint32_t encode_small_float(double a, int ebits, int mbits, int bias, double maxv, uint32_t max_pattern) {
  if (!(a > 0.0)) return 0;
  if (a >= maxv) return max_pattern;
  int e;
  std::frexp(a, &e);          // a = f * 2^e, f in [0.5, 1)
  int exp = e - 1;            // a = 1.x * 2^exp
  const int emin = 1 - bias;  // smallest normal exponent
  if (exp < emin) exp = emin; // subnormal range: fixed quantum 2^(emin - mbits)
  uint64_t k = round_to_grid(a, exp - mbits);  // k in [2^mbits, 2^(mbits+1)] for normals
  uint32_t biased;
  uint32_t frac;
  if (k >= (1ull << (mbits + 1))) {  // rounding carried into the next binade
    k >>= 1;
    exp++;
  }
  if (k < (1ull << mbits)) {  // subnormal (or rounded to zero)
    biased = 0;
    frac = (uint32_t)k;
  } else {
    biased = (uint32_t)(exp + bias);
    frac = (uint32_t)(k - (1ull << mbits));
  }
  uint32_t pat = (biased << mbits) | frac;
  return pat > max_pattern ? max_pattern : pat;
}

inline uint16_t to_fp16(double v) {
  uint16_t sign = std::signbit(v) ? 0x8000 : 0;
  if (std::isnan(v)) return 0x7e00;
  double a = std::fabs(v);
  if (a >= 65520.0) return sign | 0x7c00;  // rounds to infinity
  return sign | (uint16_t)encode_small_float(a, 5, 10, 15, 65504.0 + 16.0, 0x7bff);
}

// Rounded from the double directly (not through binary32, which could round twice).
inline uint16_t to_bf16(double v) {
  uint16_t sign = std::signbit(v) ? 0x8000 : 0;
  if (std::isnan(v)) return 0x7fc0;
  double a = std::fabs(v);
  const double boundary = std::ldexp(2.0 - 1.0 / 256.0, 127);  // halfway past the largest finite
  if (a >= boundary) return sign | 0x7f80;
  return sign | (uint16_t)encode_small_float(a, 8, 7, 127, boundary, 0x7f7f);
}

inline uint8_t to_e4m3(double v) {
  uint8_t sign = std::signbit(v) ? 0x80 : 0;
  if (std::isnan(v)) return 0x7f;
  return sign | (uint8_t)encode_small_float(std::fabs(v), 4, 3, 7, 448.0, 0x7e);
}

inline double from_fp16(uint16_t h) {
  int e = (h >> 10) & 0x1f, m = h & 0x3ff;
  double s = (h & 0x8000) ? -1.0 : 1.0;
  if (e == 0) return s * std::ldexp((double)m, -24);
  if (e == 31) return m ? NAN : s * INFINITY;
  return s * std::ldexp((double)(m | 0x400), e - 25);
}

inline double from_e4m3(uint8_t b) {
  int e = (b >> 3) & 0xf, m = b & 7;
  double s = (b & 0x80) ? -1.0 : 1.0;
  if (e == 15 && m == 7) return NAN;
  if (e == 0) return s * std::ldexp((double)m, -9);
  return s * std::ldexp((double)(m | 8), e - 10);
}

}  // namespace hmvm
