// Philox-4x32-10 counter-based generator (J. K. Salmon, M. A. Moraes,
// R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): ten rounds of two 32x32->64-bit multiplies and a Weyl key schedule.
// Shared by the kernels that draw random numbers on the device; each picks its
// own counter layout, so streams of different kernels never coincide.
#pragma once

#include <cstdint>

namespace cb2 {

// Runs the ten rounds on the counter x[0..3] with the key (k0, k1), in place.
__device__ __forceinline__ void philox4x32_10(uint32_t x[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * x[0], hi0 = __umulhi(0xD2511F53u, x[0]);
    const uint32_t lo1 = 0xCD9E8D57u * x[2], hi1 = __umulhi(0xCD9E8D57u, x[2]);
    const uint32_t y0 = hi1 ^ x[1] ^ k0, y2 = hi0 ^ x[3] ^ k1;
    x[0] = y0;
    x[1] = lo1;
    x[2] = y2;
    x[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// A double in [0, 1) with 53 random bits from the first two output words.
__device__ __forceinline__ double philox_unit(const uint32_t x[4]) {
  const uint64_t bits = ((uint64_t)x[0] << 32) | x[1];
  return (double)(bits >> 11) * 0x1.0p-53;
}

}  // namespace cb2
