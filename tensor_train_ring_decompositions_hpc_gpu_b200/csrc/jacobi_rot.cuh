// The Jacobi rotation shared by the single-matrix and the batched eigen-solvers.
#pragma once
#include <math.h>

namespace ttr {

// Whether the pair (p, q) is rotated: |a_pq| above 1e-12 of sqrt(a_pp a_qq) and above 1e-14 of
// the largest diagonal (values scaled by inv_s = 1 / that diagonal).  Eigenvalues then carry
// (1e-12)^2 relative error, residuals 1e-12 of the norm, and the solve ends about one sweep
// earlier than with a 1e-14 cut.
__device__ __forceinline__ bool jacobi_needed(double app, double aqq, double apq, double inv_s) {
  const double ps = app * inv_s, qs = aqq * inv_s, as = apq * inv_s;
  return fabs(as) > 1e-14 && as * as > 1e-24 * fabs(ps * qs);
}

// The rotation annihilating a_pq of [[a_pp, a_pq], [a_pq, a_qq]] in two halves, so that the
// latency-critical part is short: an FP32 (c, s) and an FP64 renormalisation.
//
// FP32 half: with d = a_qq - a_pp (formed in FP64, then rounded), e = 2 a_pq, h = sqrt(d^2 + e^2)
// and u = h + |d|, the smaller-angle rotation has t = sign(d) e / u, and since
// 1 + t^2 = 2 h u / u^2,
//     c = u / sqrt(2 h u),   s = sign(d) e / sqrt(2 h u),
// so two reciprocal square roots (h = x rsqrt(x)) give (c, s) with no division.  Both factors of s
// carry small relative errors, so the rotation leaves ~1e-7 |a_pq| behind however small the
// angle.  (1, 0) when the pair is not rotated.  The skip test runs in FP64 beside the FP32 path.
__device__ __forceinline__ float2 jacobi_cs32(double app, double aqq, double apq, double inv_s) {
  const double ps = app * inv_s, qs = aqq * inv_s, as = apq * inv_s;
  const bool need = fabs(as) > 1e-14 && as * as > 1e-24 * fabs(ps * qs);
  const float d = (float)(qs - ps), e = 2.0f * (float)as;
  const float x = fmaf(d, d, e * e);
  const float h = need ? x * rsqrtf(x) : 1.0f;
  const float u = h + fabsf(d);
  const float w = rsqrtf(2.0f * h * u);
  const float c = u * w, s = (d >= 0.0f ? e : -e) * w;
  return need ? make_float2(c, s) : make_float2(1.0f, 0.0f);
}

// FP64 (c, s) from the FP32 pair: with dl = c32^2 + s32^2 - 1 (the products are exact in FP64),
// scale both by 1 / sqrt(1 + dl) = 1 - dl/2 + 3 dl^2 / 8 + O(dl^3); |dl| ~ 1e-7, so the applied
// rotation is orthogonal to FP64 rounding.  (1, 0) stays (1, 0) exactly.  A solver that logs the
// FP32 pairs and replays them rebuilds bit-identical rotations with this function.
__device__ __forceinline__ void rot_from_cs32(float2 r, double& c, double& s) {
  const double c0 = r.x, s0 = r.y;
  const double dl = fma(c0, c0, fma(s0, s0, -1.0));
  const double g = fma(dl, fma(dl, 0.375, -0.5), 1.0);
  c = c0 * g;
  s = s0 * g;
}

__device__ __forceinline__ bool jacobi_rotation(double app, double aqq, double apq, double inv_s, double& c,
                                                double& s) {
  const float2 r = jacobi_cs32(app, aqq, apq, inv_s);
  rot_from_cs32(r, c, s);
  return r.y != 0.0f;
}

}  // namespace ttr
