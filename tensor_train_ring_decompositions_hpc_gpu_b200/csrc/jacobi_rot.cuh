// The Jacobi rotation shared by the single-matrix and the batched eigen-solvers.
#pragma once
#include <math.h>

namespace ttr {

// Rotation (c, s) annihilating a_pq of the 2 x 2 block [[a_pp, a_pq], [a_pq, a_qq]] (values
// scaled by inv_s for the skip test).  Returns false (c = 1, s = 0) when a_pq is negligible.
// t = sign(d) e / (|d| + sqrt(d^2 + e^2)) with d = a_qq - a_pp, e = 2 a_pq is the smaller root of
// t^2 + 2 (d / e) t - 1 = 0, formed without the quotient d / e; FP32 suffices for t.
// c = 1 / sqrt(1 + t^2) to FP64 precision: FP32 estimate, then two Newton steps
// y <- y (3 - x y^2) / 2, each squaring the relative error.
// Whether the pair (p, q) is rotated: |a_pq| above 1e-12 of sqrt(a_pp a_qq) and above 1e-14 of
// the largest diagonal (values scaled by inv_s = 1 / that diagonal).  Eigenvalues then carry
// (1e-12)^2 relative error, residuals 1e-12 of the norm, and the solve ends about one sweep
// earlier than with a 1e-14 cut.
__device__ __forceinline__ bool jacobi_needed(double app, double aqq, double apq, double inv_s) {
  const double ps = app * inv_s, qs = aqq * inv_s, as = apq * inv_s;
  return fabs(as) > 1e-14 && as * as > 1e-24 * fabs(ps * qs);
}

// The rotation in two halves: the FP32 tangent t (0 when the pair is not rotated), and (c, s)
// from t in FP64.  The large-N solver logs t per pair and round and rebuilds (c, s) from it when it
// replays the rotations on the eigenvectors: the same arithmetic gives the same bits.
__device__ __forceinline__ float jacobi_tf(double app, double aqq, double apq, double inv_s) {
  if (!jacobi_needed(app, aqq, apq, inv_s)) return 0.0f;
  const double ps = app * inv_s, qs = aqq * inv_s, as = apq * inv_s;
  const float d = (float)(qs - ps), e = 2.0f * (float)as;
  const float h = sqrtf(fmaf(d, d, e * e));
  return (d >= 0.0f ? e : -e) * __frcp_rn(fabsf(d) + h);
}

__device__ __forceinline__ void rot_from_tf(float tf, double& c, double& s) {
  const double t = (double)tf;
  const double x = fma(t, t, 1.0);
  double y = (double)rsqrtf((float)x);
  y = y * fma(-0.5 * x, y * y, 1.5);
  y = y * fma(-0.5 * x, y * y, 1.5);
  c = y;
  s = t * y;
}

__device__ __forceinline__ bool jacobi_rotation(double app, double aqq, double apq, double inv_s, double& c,
                                                double& s) {
  c = 1.0;
  s = 0.0;
  if (!jacobi_needed(app, aqq, apq, inv_s)) return false;
  rot_from_tf(jacobi_tf(app, aqq, apq, inv_s), c, s);
  return true;
}

}  // namespace ttr
