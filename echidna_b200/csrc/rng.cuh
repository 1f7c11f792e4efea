// Counter-based random numbers for the device (directions and coordinate samples).
#pragma once
#include <stdint.h>

namespace ech {

// Philox-4x32-10 (Salmon et al., SC'11) keyed by `seed`; counter (point, dir, i).
__device__ __forceinline__ uint32_t philox_bits(uint64_t seed, uint64_t point, uint32_t dir, uint32_t i) {
  uint32_t c0 = (uint32_t)point, c1 = (uint32_t)(point >> 32), c2 = dir, c3 = i;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c0;
}

// Uniform in [0, 1) with 24 random bits.
__device__ __forceinline__ float philox_uniform(uint64_t seed, uint64_t point, uint32_t dir, uint32_t i) {
  return (float)(philox_bits(seed, point, dir, i) >> 8) * (1.0f / 16777216.0f);
}

}  // namespace ech
