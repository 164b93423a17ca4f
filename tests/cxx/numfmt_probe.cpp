// Exposes the planner's storage-format encoders (csrc/numfmt.hpp) to the
// tests: probe_encode(type, src, dst, n) with type 2 FP16, 3 FP8 E4M3, 4 BF16.
#include <cstdint>

#include "numfmt.hpp"

extern "C" void probe_encode(int type, const double* src, void* dst, long n) {
  for (long i = 0; i < n; i++) {
    if (type == 2) static_cast<uint16_t*>(dst)[i] = hmvm::to_fp16(src[i]);
    else if (type == 4) static_cast<uint16_t*>(dst)[i] = hmvm::to_bf16(src[i]);
    else static_cast<uint8_t*>(dst)[i] = hmvm::to_e4m3(src[i]);
  }
}
