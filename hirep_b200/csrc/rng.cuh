// rng.cuh -- the device random-number generator behind gaussian_momenta and
// gaussian_spinor_field.
//
// HiRep draws momenta and pseudofermion sources with ranlux on the host
// (LibHR/Random/ranlxd.c, gauss.c).  Here every number is a pure function of
// (key, stream, element index) through the counter-based generator
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC11: ten rounds of two 32x32->64-bit multiplies with the
// multipliers 0xD2511F53 and 0xCD9E8D57, the key bumped by the Weyl constants
// 0x9E3779B9 and 0xBB67AE85 between rounds), so one kernel pass draws a whole
// field with no generator state in memory.  One Philox block gives two
// uniforms of 53 bits in (0, 1), and the Box-Muller transform turns them into
// two independent standard Gaussians.  The numbers differ from HiRep's ranlux
// ones; their distribution is the same.
#pragma once
#include <stdint.h>

namespace hrgpu {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, n3 = (uint32_t)p0;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// two standard Gaussians from the Philox block (q, stream) under key (k0, k1)
__device__ __forceinline__ double2 gauss_pair(uint64_t q, uint64_t stream, uint32_t k0, uint32_t k1) {
  uint32_t c[4] = {(uint32_t)q, (uint32_t)(q >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  philox4x32_10(c, k0, k1);
  const double u1 = ((double)((((uint64_t)c[0] << 32) | c[1]) >> 11) + 0.5) * 0x1p-53;  // (0, 1)
  const double u2 = ((double)((((uint64_t)c[2] << 32) | c[3]) >> 11) + 0.5) * 0x1p-53;
  const double r = sqrt(-2.0 * log(u1));
  double s, co;
  sincospi(2.0 * u2, &s, &co);
  return make_double2(r * co, r * s);
}

}  // namespace hrgpu
