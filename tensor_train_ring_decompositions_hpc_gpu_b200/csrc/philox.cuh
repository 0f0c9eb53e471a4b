// Philox4x32-10 counter-based generator (Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC 2011): 10 rounds of the 4x32 Philox S-box with the published multipliers and
// Weyl key increments.  Shared by the Gaussian test-matrix kernels.
#pragma once
#include <cstdint>

namespace ttr {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Four N(0,1) values from one Philox call (Box-Muller on the two word pairs, with the hardware
// approximations: absolute error ~1e-6; the angle is taken in [-pi, pi)).
__device__ __forceinline__ float4 philox_normal4(unsigned long long call, unsigned stream, unsigned long long seed) {
  const uint4 w = philox4x32_10(make_uint4((unsigned)(call & 0xFFFFFFFFull), stream, (unsigned)(call >> 32), 0u),
                                make_uint2((unsigned)(seed & 0xFFFFFFFFull), (unsigned)(seed >> 32)));
  const float sc = 2.3283064365386963e-10f;  // 2^-32
  const float u0 = ((float)w.x + 0.5f) * sc, u1 = ((float)w.y + 0.5f) * sc;
  const float u2 = ((float)w.z + 0.5f) * sc, u3 = ((float)w.w + 0.5f) * sc;
  const float r0 = sqrtf(-2.0f * __logf(u0)), r1 = sqrtf(-2.0f * __logf(u2));
  float s0, c0, s1, c1;
  __sincosf(6.283185307179586f * (u1 - 0.5f), &s0, &c0);
  __sincosf(6.283185307179586f * (u3 - 0.5f), &s1, &c1);
  return make_float4(-r0 * c0, -r0 * s0, -r1 * c1, -r1 * s1);
}

}  // namespace ttr
