// packed4.cuh -- expansion of packed 4+4-bit complex samples to int8.
//
// A packed byte holds one complex sample: the real part in the high nibble,
// the imaginary part in the low nibble, both 4-bit two's complement.  It
// expands to the two int8 bytes {re, im} of the [t][f][s][p][c] layout.
#pragma once

#include <stdint.h>

namespace xgpu {

// Four packed samples (one 32-bit word) -> eight int8 bytes in the same order.
// Byte-wise: a nibble v in 0..15 is the signed value (v ^ 8) - 8.
__device__ __forceinline__ uint2 expand_packed4(uint32_t w) {
  const uint32_t re = __vsub4(((w >> 4) & 0x0F0F0F0Fu) ^ 0x08080808u, 0x08080808u);
  const uint32_t im = __vsub4((w & 0x0F0F0F0Fu) ^ 0x08080808u, 0x08080808u);
  return make_uint2(__byte_perm(re, im, 0x5140), __byte_perm(re, im, 0x7362));
}

}  // namespace xgpu
