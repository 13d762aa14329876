// Counter-based random numbers shared by every generator of the library (and
// restated bit for bit in the CPU oracle): each value is a pure function of
// (seed, stream, counter).
#pragma once

#include <stdint.h>

namespace xt {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // splitmix64 output function (Steele, Lea, Flood 2014)
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}

__host__ __device__ __forceinline__ uint64_t crand(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t k = mix64(seed * 0x9e3779b97f4a7c15ULL + stream + 0x632be59bd9b4e019ULL);
  return mix64(k ^ (ctr * 0x9e3779b97f4a7c15ULL + 0xd1b54a32d192ed03ULL));
}

// bijection on [0, 2^bits): odd multiplies, xor constants and right
// xorshifts are each invertible modulo 2^bits
__host__ __device__ __forceinline__ uint64_t perm_bits(uint64_t x, int bits, uint64_t seed) {
  const uint64_t mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
  const int sh = (bits + 1) / 2;
  x &= mask;
  for (int r = 0; r < 4; r++) {
    uint64_t k = mix64(seed + 0x9e3779b97f4a7c15ULL * uint64_t(r + 1));
    x = (x * (k | 1ULL)) & mask;
    x ^= (k >> 17) & mask;
    x ^= x >> sh;
  }
  return x & mask;
}

}  // namespace xt
