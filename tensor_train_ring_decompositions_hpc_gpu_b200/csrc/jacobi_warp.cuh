// Symmetric eigen-solvers shared by the single-matrix and the batched kernels: the Jacobi
// rotation and a one-warp cyclic Jacobi for N <= 32 whose matrix never leaves the registers.
#pragma once
#include <math.h>

namespace ttr {

// Rotation (c, s) annihilating a_pq of the 2 x 2 block [[a_pp, a_pq], [a_pq, a_qq]] (values
// scaled by inv_s for the skip test).  Returns false (c = 1, s = 0) when a_pq is negligible.
// t = sign(d) e / (|d| + sqrt(d^2 + e^2)) with d = a_qq - a_pp, e = 2 a_pq is the smaller root of
// t^2 + 2 (d / e) t - 1 = 0, formed without the quotient d / e; FP32 suffices for t.
// c = 1 / sqrt(1 + t^2) to FP64 precision: FP32 estimate, then two Newton steps
// y <- y (3 - x y^2) / 2, each squaring the relative error.
__device__ __forceinline__ bool jacobi_rotation(double app, double aqq, double apq, double inv_s, double& c,
                                                double& s) {
  const double ps = app * inv_s, qs = aqq * inv_s, as = apq * inv_s;
  c = 1.0;
  s = 0.0;
  if (!(fabs(as) > 1e-15 && as * as > 1e-28 * fabs(ps * qs))) return false;
  const float d = (float)(qs - ps), e = 2.0f * (float)as;
  const float h = sqrtf(fmaf(d, d, e * e));
  const float tf = (d >= 0.0f ? e : -e) * __frcp_rn(fabsf(d) + h);
  const double t = (double)tf;
  const double x = fma(t, t, 1.0);
  double y = (double)rsqrtf((float)x);
  y = y * fma(-0.5 * x, y * y, 1.5);
  y = y * fma(-0.5 * x, y * y, 1.5);
  c = y;
  s = t * y;
  return true;
}

// Eigen-decomposition of the symmetric part of an N x N matrix (N <= 32) by ONE warp.
//
// Cyclic Jacobi with the XOR tournament: round r (r = 1..31) pairs index i with i ^ r, so over a
// sweep every pair meets exactly once and no row or column ever moves.  Lane i keeps row i of W
// in registers, XOR-swizzled: w[k] = W[i][i ^ k].  Then the diagonal is w[0], the entry of the
// round-r pair is w[r], the partner row's entry in column i ^ k is register k ^ r of lane i ^ r
// (one shuffle), and the column pair (i ^ k, i ^ k ^ r) is the register pair (k, k ^ r) with its
// rotation held by lane i ^ k.  Every index is a compile-time register number once the round
// loop is unrolled.  Each round applies W' = J^T W J (rows, then columns) and V' = V J; V is
// kept the same way in registers (VREG) or in shared memory (vsm, row stride 33 doubles).
// Indices >= N are zero rows and columns: their rotations are skipped.
//
// W element (a, b) is read at W[a * ldr + b * ldc] and symmetrised.  Output: evals[0..N)
// descending, eigenvector of evals[q] in evecs[i + ldv * q] (i < N).  Returns the sweep count,
// max_sweeps + 1 when the last sweep still rotated.  All 32 lanes of the warp must call it.
template <bool VREG>
__device__ int warp_jacobi32(const double* __restrict__ W, long long ldr, long long ldc, int N, double* vsm,
                             int max_sweeps, double* __restrict__ evals, double* __restrict__ evecs, long long ldv) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool live = lane < N;
  double w[32];
  double vr[VREG ? 32 : 1];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int j = lane ^ k;
    w[k] = (live && j < N) ? 0.5 * (W[lane * ldr + j * ldc] + W[j * ldr + lane * ldc]) : 0.0;
    if (VREG) {
      vr[VREG ? k : 0] = k == 0 ? 1.0 : 0.0;
    } else {
      vsm[lane * 33 + k] = k == 0 ? 1.0 : 0.0;
    }
  }
  double dm = fabs(w[0]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dm = fmax(dm, __shfl_xor_sync(FULL, dm, o));
  const double inv_s = dm > 0.0 ? 1.0 / dm : 1.0;
  __syncwarp();

  int sweep = 0;
  bool conv = false;
  for (; sweep < max_sweeps; ++sweep) {
    int rot = 0;
#pragma unroll
    for (int r = 1; r < 32; ++r) {
      const bool isp = lane < (lane ^ r);
      const double dpart = __shfl_xor_sync(FULL, w[0], r);
      const double off = 0.5 * (w[r] + __shfl_xor_sync(FULL, w[r], r));
      double c, s;
      if (jacobi_rotation(isp ? w[0] : dpart, isp ? dpart : w[0], off, inv_s, c, s)) rot = 1;
      // rows: new row p = c row_p - s row_q, new row q = s row_p + c row_q
      const double sr = isp ? -s : s;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int k2 = k ^ r;
        if (k < k2) {
          const double pk = __shfl_xor_sync(FULL, w[k2], r);
          const double pk2 = __shfl_xor_sync(FULL, w[k], r);
          w[k] = fma(c, w[k], sr * pk);
          w[k2] = fma(c, w[k2], sr * pk2);
        }
      }
      // columns (and V): new col p = c col_p - s col_q, new col q = s col_p + c col_q
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int k2 = k ^ r;
        if (k < k2) {
          const double cj = __shfl_xor_sync(FULL, c, k);
          const double sj = __shfl_xor_sync(FULL, s, k);
          const double sg = ((lane ^ k) < (lane ^ k2)) ? sj : -sj;
          const double a = w[k], b = w[k2];
          w[k] = fma(cj, a, -sg * b);
          w[k2] = fma(cj, b, sg * a);
          if (VREG) {
            const double va = vr[VREG ? k : 0], vb = vr[VREG ? k2 : 0];
            vr[VREG ? k : 0] = fma(cj, va, -sg * vb);
            vr[VREG ? k2 : 0] = fma(cj, vb, sg * va);
          } else {
            const double va = vsm[lane * 33 + k], vb = vsm[lane * 33 + k2];
            vsm[lane * 33 + k] = fma(cj, va, -sg * vb);
            vsm[lane * 33 + k2] = fma(cj, vb, sg * va);
          }
        }
      }
    }
    if (!__any_sync(FULL, rot)) {
      conv = true;
      ++sweep;
      break;
    }
  }
  // descending order (NaN last, ties by index)
  double la = live ? w[0] : -INFINITY;
  if (la != la) la = -INFINITY;
  int rank = 0;
  for (int b = 0; b < 32; ++b) {
    double lb = __shfl_sync(FULL, la, b);
    rank += (b < N && (lb > la || (lb == la && b < lane))) ? 1 : 0;
  }
  if (live) evals[rank] = w[0];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int j = lane ^ k;
    const int rj = __shfl_xor_sync(FULL, rank, k);
    const double v = VREG ? vr[VREG ? k : 0] : vsm[lane * 33 + k];
    if (live && j < N) evecs[lane + ldv * rj] = v;
  }
  __syncwarp();
  return conv ? sweep : max_sweeps + 1;
}

}  // namespace ttr
