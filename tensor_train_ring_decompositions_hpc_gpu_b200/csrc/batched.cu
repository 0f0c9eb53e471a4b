// Batched TT-SVD of many small tensors in one persistent launch.
//
// One CTA decomposes one tensor at a time and takes the next tensor index from a global work
// counter, so the SMs stay busy whatever the size mix.  Every step of a tensor runs inside the
// CTA: the exact Gram-eigen step when the small side of the unfolding is <= 32 (Gram in FP64,
// Jacobi in shared memory), otherwise EDrSVD (Philox Gaussian sketch generated on the fly, both
// CholeskyQR passes in shared memory, projection B = Q^T A with the Gram B B^T accumulated
// alongside, Jacobi).  Ranks follow the delta-truncation rule of tt_svd (eps > 0) or are the
// largest allowed (eps = 0), capped by rmax.  The unfoldings of the tensor being processed
// live in a per-CTA scratch (ping-pong), cores are written compactly in the caller's buffer.
// The reference decomposes one tensor per call (ttdec_gpu_float, ttdec_half_lu_device_6) and
// has no batched path.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"
#include "philox.cuh"
#include "bl_solver.cuh"

namespace ttr {
namespace {

constexpr int BT = 512;       // threads per CTA
constexpr int BMAXM = 512;    // largest row count of a randomized unfolding
constexpr int BSMALL = 32;    // largest exact small side / sketch width
constexpr int BMAXD = 8;      // largest order
// Tunable: columns of the Gaussian test matrix generated per chunk of the sketch (BCH, a
// template parameter) and the order in which the work counter hands out tensors.
constexpr int kChunks[3] = {16, 32, 64};
enum { SCHED_NATURAL = 0, SCHED_LARGEST_FIRST = 1 };

struct BatchShape {
  int d;
  int n[BMAXD];
  long long size;
  long long x_off;
  long long core_off;
};

// Shared-memory layout of the kernel (bytes).
constexpr size_t SM_CHUNK = (size_t)BMAXM * BSMALL * sizeof(float);         // U (m x r)
constexpr size_t SM_YQ = (size_t)BMAXM * (BSMALL + 1) * sizeof(float);        // Y, Q (stride ks|1)
constexpr size_t SM_W = (size_t)BSMALL * BSMALL * sizeof(double);             // Gram
constexpr size_t SM_JAC = 2 * (size_t)BSMALL * BSMALL * sizeof(double);       // Jacobi buffers
constexpr size_t SM_RED = (size_t)BT * 2 * sizeof(double);                    // reductions
template <int BCH>
constexpr size_t sm_om() { return (size_t)BCH * BSMALL * sizeof(float); }   // Omega chunk
template <int BCH>
constexpr size_t sm_total() { return SM_CHUNK + SM_YQ + SM_W + SM_JAC + sm_om<BCH>() + SM_RED + 1024; }

struct Smem {
  float* chunk;   // BMAXM x BSMALL
  float* yq;      // BMAXM x (BSMALL+1)
  double* w;      // BSMALL x BSMALL (row-major, stride Np)
  double* jac;    // 2 x BSMALL^2 (the eigen-solver's double-buffered W)
  float* om;      // BCH x BSMALL
  double* red;    // 2 * BT
};

__device__ double cta_sum(double v, double* red) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < BT / 32; ++w) t += red[w];
  __syncthreads();
  return t;
}

// W (N x N, row-major, stride N) = sum over `nvec` vectors of v v^T, where component p of
// vector j is at base[p * ps + j * vs] (N <= BSMALL).  4 x 4 register tiles of the upper
// triangle, vectors split into groups of threads, groups added in order through W.
// F32P: products of the FP32 data summed in FP32 over 64 vectors of a thread, then in FP64 (the
// Grams that feed an eigen-solve: relative errors ~1e-8 of the entries, and no FP64 conversion
// per product); otherwise FP64 products (CholeskyQR of a sketch, whose condition number the
// Gram squares).
template <bool F32P>
__device__ void cta_gram(const float* __restrict__ base, long long ps, long long vs, int N, long long nvec,
                         double* W) {
  const int tid = threadIdx.x;
  const int TT = (N + 3) / 4;
  const int nt = TT * (TT + 1) / 2;
  const int groups = min(32, max(1, BT / nt));
  const int t = tid % nt, g = tid / nt;
  const bool act = g < groups;
  int ta = 0, rem = act ? t : 0;
  while (rem >= TT - ta) {
    rem -= TT - ta;
    ++ta;
  }
  const int tb = ta + rem;
  double acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = 0.0;
  if (act) {
    float accf[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) accf[e] = 0.f;
    int cnt = 0;
    for (long long j = g; j < nvec; j += groups) {
      float a[4], b[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int ia = 4 * ta + p, ib = 4 * tb + p;
        a[p] = ia < N ? base[ia * ps + j * vs] : 0.f;
        b[p] = ib < N ? base[ib * ps + j * vs] : 0.f;
      }
      if constexpr (F32P) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) accf[p * 4 + q] = fmaf(a[p], b[q], accf[p * 4 + q]);
        if (++cnt == 64) {
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            acc[e] += (double)accf[e];
            accf[e] = 0.f;
          }
          cnt = 0;
        }
      } else {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p * 4 + q] = fma((double)a[p], (double)b[q], acc[p * 4 + q]);
      }
    }
    if constexpr (F32P) {
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[e] += (double)accf[e];
    }
  }
  for (int gg = 0; gg < groups; ++gg) {
    if (act && g == gg) {
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = 4 * ta + p, j = 4 * tb + q;
          if (i < N && j < N && i <= j) {  // upper triangle, mirrored (diagonal tiles hold both halves)
            const double v = (gg == 0 ? 0.0 : W[i * N + j]) + acc[p * 4 + q];
            W[i * N + j] = v;
            if (i != j) W[j * N + i] = v;
          }
        }
    }
    __syncthreads();
  }
}

template <int W>
struct Width {
  static constexpr int value = W;
};

// Calls f(Width<W>{}) with W = n rounded up to a multiple of 8 (n <= BSMALL).  The per-column
// register loops of a step (a rank or sketch width of 2..32) then run over W columns rather than
// all BSMALL with most of them predicated off; columns beyond n are computed on zeros or ignored
// and never stored, so every kept column's FMA sequence is the same whatever W is.
template <class F>
__device__ __forceinline__ void by_width(int n, F&& f) {
  if (n <= 8) f(Width<8>{});
  else if (n <= 16) f(Width<16>{});
  else if (n <= 24) f(Width<24>{});
  else f(Width<32>{});
}

// Largest-|entry| of each of the first r columns of U (rows x r, stride ld) made positive;
// the sign is recorded in sgn[c] (+1/-1) and applied to U.
__device__ void cta_canon(float* U, int rows, int ld, int r, float* sgn) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = warp; c < r; c += BT / 32) {
    float best = 0.f;
    int bi = rows;
    for (int i = lane; i < rows; i += 32) {
      const float v = fabsf(U[i + (long long)ld * c]);
      if (v > best || (v == best && i < bi)) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    const float s = (bi < rows && U[bi + (long long)ld * c] < 0.f) ? -1.f : 1.f;
    for (int i = lane; i < rows; i += 32) U[i + (long long)ld * c] *= s;
    if (lane == 0) sgn[c] = s;
  }
  __syncthreads();
}

// Rank from eigenvalues (descending) of an unfolding whose energy is `energy`: the smallest r
// (<= cap) whose discarded energy is <= delta2; eps = 0 keeps cap.  Returns r and updates the
// energy carried and the discarded total.
__device__ int pick_rank(const double* lam, int nev, int cap, double delta2, bool adaptive, double energy,
                         double* kept_out, double* tail_out) {
  int r = 0;
  double kept = 0.0;
  if (!adaptive) {
    for (; r < cap; ++r) kept += fmax(lam[r], 0.0);
  } else {
    while (r < cap && (r == 0 || energy - kept > delta2)) kept += fmax(lam[r++], 0.0);
  }
  (void)nev;
  *kept_out = kept;
  *tail_out = fmax(energy - kept, 0.0);
  return r;
}

template <int BCH>
__global__ void __launch_bounds__(BT, 1)
    k_tt_batched(const BatchShape* __restrict__ shp, const int* __restrict__ order, int count,
                 const float* __restrict__ x,
                 float* __restrict__ cores, int* __restrict__ ranks_out, double* __restrict__ err_out,
                 float* __restrict__ scratch, long long scratch_per_cta, long long half, double eps, int rmax,
                 int oversample, unsigned long long seed, int max_sweeps, int* __restrict__ counter,
                 DevStatus* st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Smem S;
  {
    unsigned char* p = smraw;
    S.chunk = reinterpret_cast<float*>(p);
    p += SM_CHUNK;
    S.yq = reinterpret_cast<float*>(p);
    p += SM_YQ;
    S.w = reinterpret_cast<double*>(p);
    p += SM_W;
    S.jac = reinterpret_cast<double*>(p);
    p += SM_JAC;
    S.om = reinterpret_cast<float*>(p);
    p += sm_om<BCH>();
    S.red = reinterpret_cast<double*>(p);
  }
  __shared__ double lam[BSMALL], evec[BSMALL * BSMALL];
  __shared__ float sgn[BSMALL], sig_inv[BSMALL];
  __shared__ int sh_i[4];
  const int tid = threadIdx.x;
  float* buf0 = scratch + (long long)blockIdx.x * scratch_per_cta;
  float* buf1 = buf0 + half;
  float* Bg = buf1 + half;  // ks x cols of the randomized steps

  for (;;) {
    if (tid == 0) sh_i[0] = atomicAdd(counter, 1);
    __syncthreads();
    const int slot = sh_i[0];
    __syncthreads();
    if (slot >= count) break;
    const int t = order ? order[slot] : slot;
    const BatchShape sh = shp[t];
    const int d = sh.d;
    const float* src = x + sh.x_off;
    float* cp = cores + sh.core_off;
    long long size = sh.size;
    // ||X||^2
    double s2 = 0.0;
    for (long long i = tid; i < size; i += BT) s2 = fma((double)src[i], (double)src[i], s2);
    const double xn2 = cta_sum(s2, S.red);
    const bool adaptive = eps > 0.0;
    const double delta2 = eps * eps * xn2 / (double)max(d - 1, 1);
    double energy = xn2, tails = 0.0;
    int r_prev = 1;
    if (tid == 0) ranks_out[(long long)t * (BMAXD + 1)] = 1;
    bool fail = false;
    for (int k = 0; k < d - 1 && !fail; ++k) {
      const long long m = (long long)r_prev * sh.n[k];
      const long long cols = size / m;
      const long long small = m < cols ? m : cols;
      const int cap = (int)min((long long)rmax, small);
      float* dst = (k & 1) ? buf0 : buf1;
      int r = 1;
      if (small <= BSMALL) {
        // ---- exact Gram-eigen step ----
        const int N = (int)small;
        if (m <= cols) cta_gram<true>(src, 1, m, N, cols, S.w);   // W = A A^T, vectors = columns
        else cta_gram<true>(src, m, 1, N, m, S.w);                // W = A^T A, vectors = rows
        const int sw = bl_solve<0>(S.w, N, lam, evec, max_sweeps, S.jac);
        if (tid == 0 && st) {
          atomicMax(&st->sweeps, sw);
          if (sw > max_sweeps) dev_fail(st, TT_ERR_NOCONV, t);
        }
        double full = 0.0;
        for (int i = 0; i < N; ++i) full += fmax(lam[i], 0.0);
        double kept, tail;
        r = pick_rank(lam, N, cap, delta2, adaptive, adaptive ? full : energy, &kept, &tail);
        tails += tail;
        energy = kept;
        if (m <= cols) {
          // U = E_r (m x r): canonical signs, core, next = U^T A (r x cols, column-major)
          float* U = S.chunk;  // m x r
          for (int idx = tid; idx < (int)m * r; idx += BT) U[idx] = (float)evec[(idx % m) + m * (idx / m)];
          __syncthreads();
          cta_canon(U, (int)m, (int)m, r, sgn);
          for (int idx = tid; idx < (int)m * r; idx += BT) cp[idx] = U[idx];
          by_width(r, [&](auto w) {
            constexpr int W = decltype(w)::value;
            float* Ut = S.yq;  // U row-major (m x W, zero beyond r): a row's columns in W/4 float4 loads
            for (int idx = tid; idx < (int)m * W; idx += BT) {
              const int i = idx / W, c = idx - i * W;
              Ut[idx] = c < r ? U[i + m * c] : 0.f;
            }
            __syncthreads();
            for (long long j = tid; j < cols; j += BT) {
              uint64_t acc2[W / 2];  // columns (2c, 2c+1) as FP32 pairs (fma.rn.f32x2 per pair)
#pragma unroll
              for (int c = 0; c < W / 2; ++c) acc2[c] = 0ull;
              const float* a = src + j * m;
              for (int i = 0; i < (int)m; ++i) {
                const uint64_t av2 = f2_dup(a[i]);
                const ulonglong2* u2 = reinterpret_cast<const ulonglong2*>(Ut + i * W);
#pragma unroll
                for (int c4 = 0; c4 < W / 4; ++c4) {
                  const ulonglong2 u = u2[c4];
                  ffma2(acc2[2 * c4 + 0], av2, u.x);
                  ffma2(acc2[2 * c4 + 1], av2, u.y);
                }
              }
#pragma unroll
              for (int c2 = 0; c2 < W / 2; ++c2) {
                float lo, hi;
                f2_unpack(acc2[c2], lo, hi);
                if (2 * c2 < r) dst[j * r + 2 * c2] = lo;
                if (2 * c2 + 1 < r) dst[j * r + 2 * c2 + 1] = hi;
              }
            }
          });
        } else {
          // cols <= 32 < m: V (cols x cols), U = A V_r / sigma (m x r), next = sigma V_r^T
          for (int c = tid; c < r; c += BT) sig_inv[c] = lam[c] > 0.0 ? (float)(1.0 / sqrt(lam[c])) : 0.f;
          const int nc = (int)cols;
          by_width(nc, [&](auto w) {
            constexpr int W = decltype(w)::value;
            float* Vf = S.chunk;  // Vf[c W + q] = V[q][c] in FP32 (zero beyond nc)
            for (int idx = tid; idx < r * W; idx += BT) {
              const int c = idx / W, q = idx - c * W;
              Vf[idx] = q < nc ? (float)evec[q + nc * c] : 0.f;
            }
            __syncthreads();
            for (long long i = tid; i < m; i += BT) {
              float arow[W];
#pragma unroll
              for (int q = 0; q < W; ++q) arow[q] = q < nc ? src[i + m * q] : 0.f;
              for (int c = 0; c < r; ++c) {
                const float4* v4 = reinterpret_cast<const float4*>(Vf + c * W);
                float acc = 0.f;
#pragma unroll
                for (int q4 = 0; q4 < W / 4; ++q4) {
                  const float4 v = v4[q4];
                  if (4 * q4 + 0 < nc) acc = fmaf(arow[4 * q4 + 0], v.x, acc);
                  if (4 * q4 + 1 < nc) acc = fmaf(arow[4 * q4 + 1], v.y, acc);
                  if (4 * q4 + 2 < nc) acc = fmaf(arow[4 * q4 + 2], v.z, acc);
                  if (4 * q4 + 3 < nc) acc = fmaf(arow[4 * q4 + 3], v.w, acc);
                }
                cp[i + m * c] = acc * sig_inv[c];
              }
            }
          });
          __syncthreads();
          // canonical signs on the core columns (global memory), mirrored on the rows of sigma V^T
          cta_canon(cp, (int)m, (int)m, r, sgn);
          for (int idx = tid; idx < r * nc; idx += BT) {
            const int c = idx % r, q = idx / r;  // dst column-major r x cols: dst[c + r q]
            dst[idx] = sgn[c] * (float)(sqrt(fmax(lam[c], 0.0)) * evec[q + nc * c]);
          }
        }
      } else if (m <= BMAXM) {
        // ---- randomized step (EDrSVD) ----
        const int ks = (int)min((long long)min(cap + oversample, BSMALL), small);
        const int SY = ks | 1;  // odd row stride of Y / Q in shared memory
        const int mi = (int)m;
        // Y = A Omega, Omega (cols x ks) N(0,1) from Philox: element (j, c) is component j & 3 of
        // call (c * cols4 + (j & ~3)) / 4, cols4 = cols rounded up to a multiple of 4.
        const long long cols4 = (cols + 3) & ~3LL;
        const unsigned stream = (unsigned)(t * BMAXD + k);
        by_width(ks, [&](auto w) {
          constexpr int W = decltype(w)::value;
          uint64_t yacc2[W / 2];  // sketch columns (2c, 2c+1) as FP32 pairs
#pragma unroll
          for (int c = 0; c < W / 2; ++c) yacc2[c] = 0ull;
          for (long long j0 = 0; j0 < cols; j0 += BCH) {
            const int nj = (int)min((long long)BCH, cols - j0);
            __syncthreads();
            for (int q = tid; q < (BCH / 4) * W; q += BT) {
              const int c = q / (BCH / 4), j4 = 4 * (q % (BCH / 4));
              // columns ks..W-1 of the chunk are zero: their accumulators stay finite and unused
              const float4 g = c < ks
                                   ? philox_normal4((unsigned long long)((c * cols4 + j0 + j4) >> 2), stream, seed)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
              S.om[(j4 + 0) * BSMALL + c] = g.x;
              S.om[(j4 + 1) * BSMALL + c] = g.y;
              S.om[(j4 + 2) * BSMALL + c] = g.z;
              S.om[(j4 + 3) * BSMALL + c] = g.w;
            }
            __syncthreads();
            if (tid < mi) {
              for (int jj = 0; jj < nj; ++jj) {
                const uint64_t av2 = f2_dup(src[tid + m * (j0 + jj)]);
                const ulonglong2* o2 = reinterpret_cast<const ulonglong2*>(S.om + jj * BSMALL);
#pragma unroll
                for (int c4 = 0; c4 < W / 4; ++c4) {
                  const ulonglong2 o = o2[c4];
                  ffma2(yacc2[2 * c4 + 0], av2, o.x);
                  ffma2(yacc2[2 * c4 + 1], av2, o.y);
                }
              }
            }
          }
          __syncthreads();
          if (tid < mi)
#pragma unroll
            for (int c2 = 0; c2 < W / 2; ++c2) {
              float lo, hi;
              f2_unpack(yacc2[c2], lo, hi);
              if (2 * c2 < ks) S.yq[tid * SY + 2 * c2] = lo;
              if (2 * c2 + 1 < ks) S.yq[tid * SY + 2 * c2 + 1] = hi;
            }
        });
        __syncthreads();
        // CholeskyQR2 on Y (rows x ks in shared memory): Gram in FP64, Cholesky, substitution
        for (int pass = 0; pass < 2; ++pass) {
          cta_gram<false>(S.yq, 1, SY, ks, mi, S.w);
          double* Wc = S.w;
          double dmax = 0.0;
          for (int i = 0; i < ks; ++i) dmax = fmax(dmax, Wc[i * ks + i]);
          const double tol = 1e-12 * dmax;
          __syncthreads();  // every thread has read the diagonal before the first update changes it
          for (int kk = 0; kk < ks; ++kk) {
            const double dk = Wc[kk * ks + kk];
            if (dk > tol && dmax > 0.0) {
              const double inv = 1.0 / dk;
              const int j = kk + 1 + (tid & 31);
              if (j < ks) {
                const double wkj = Wc[kk * ks + j] * inv;
                for (int i = kk + 1 + (tid >> 5); i <= j; i += BT / 32) Wc[i * ks + j] -= Wc[kk * ks + i] * wkj;
              }
            }
            __syncthreads();
          }
          // R in FP32 once (the eigen-solver's buffer is free here): rf[k ks + c] = W[k][c] /
          // sqrt(W[k][k]) for live rows k < c (0 on dead ones), rf[ks ks + c] = 1 / sqrt(W[c][c])
          // (0: dead column), so the substitution below is FMAs only.
          float* rf = reinterpret_cast<float*>(S.jac);
          for (int idx = tid; idx < ks * ks + ks; idx += BT) {
            if (idx < ks * ks) {
              const int kk = idx / ks, c = idx - kk * ks;
              const double dk = Wc[kk * ks + kk];
              rf[idx] = (kk < c && dk > tol && dmax > 0.0) ? (float)(Wc[kk * ks + c] / sqrt(dk)) : 0.f;
            } else {
              const double dc = Wc[(idx - ks * ks) * (ks + 1)];
              rf[idx] = (dc > tol && dmax > 0.0) ? (float)(1.0 / sqrt(dc)) : 0.f;
            }
          }
          __syncthreads();
          // row i: q R = y (forward substitution; a dead column's entry is 0, so it adds nothing)
          if (tid < mi) {
            float* yr = S.yq + tid * SY;
            for (int c = 0; c < ks; ++c) {
              const float dv = rf[ks * ks + c];
              float a = yr[c];
              for (int kk = 0; kk < c; ++kk) a = fmaf(-yr[kk], rf[kk * ks + c], a);
              yr[c] = dv == 0.f ? 0.f : a * dv;
            }
          }
          __syncthreads();
        }
        // B = Q^T A (ks x cols, column-major in Bg), then W = B B^T in FP64
        by_width(ks, [&](auto w) {
          constexpr int W = decltype(w)::value;
          float* Qc = S.chunk;  // Q row-major (mi x W, zero beyond ks): a row in W/4 float4 loads
          for (int idx = tid; idx < mi * W; idx += BT) {
            const int i = idx / W, c = idx - i * W;
            Qc[idx] = c < ks ? S.yq[i * SY + c] : 0.f;
          }
          __syncthreads();
          for (long long j = tid; j < cols; j += BT) {
            uint64_t b2[W / 2];  // rows (2c, 2c+1) of B as FP32 pairs
#pragma unroll
            for (int c = 0; c < W / 2; ++c) b2[c] = 0ull;
            const float* a = src + j * m;
            for (int i = 0; i < mi; ++i) {
              const uint64_t av2 = f2_dup(a[i]);
              const ulonglong2* q2 = reinterpret_cast<const ulonglong2*>(Qc + i * W);
#pragma unroll
              for (int c4 = 0; c4 < W / 4; ++c4) {
                const ulonglong2 q = q2[c4];
                ffma2(b2[2 * c4 + 0], av2, q.x);
                ffma2(b2[2 * c4 + 1], av2, q.y);
              }
            }
#pragma unroll
            for (int c2 = 0; c2 < W / 2; ++c2) {
              float lo, hi;
              f2_unpack(b2[c2], lo, hi);
              if (2 * c2 < ks) Bg[j * ks + 2 * c2] = lo;
              if (2 * c2 + 1 < ks) Bg[j * ks + 2 * c2 + 1] = hi;
            }
          }
        });
        __syncthreads();
        cta_gram<true>(Bg, 1, ks, ks, cols, S.w);  // W = B B^T (vectors = columns of B)
        const int sw = bl_solve<0>(S.w, ks, lam, evec, max_sweeps, S.jac);
        if (tid == 0 && st) {
          atomicMax(&st->sweeps, sw);
          if (sw > max_sweeps) dev_fail(st, TT_ERR_NOCONV, t);
        }
        double kept, tail;
        r = pick_rank(lam, ks, min(cap, ks), delta2, adaptive, energy, &kept, &tail);
        tails += tail;
        energy = kept;
        // U = Q E_r (m x r) -> canonical signs -> core; next = E_r^T B with the same signs
        by_width(ks, [&](auto w) {
          constexpr int W = decltype(w)::value;
          // E_r in FP32, Ef[c W + q] = E[q][c] (zero beyond ks), in the eigen-solver's buffer
          float* Ef = reinterpret_cast<float*>(S.jac);
          for (int idx = tid; idx < r * W; idx += BT) {
            const int c = idx / W, q = idx - c * W;
            Ef[idx] = q < ks ? (float)evec[q + ks * c] : 0.f;
          }
          __syncthreads();
          float* U = S.chunk;
          for (int idx = tid; idx < mi * r; idx += BT) {
            const int i = idx % mi, c = idx / mi;
            float acc = 0.f;
            for (int q = 0; q < ks; ++q) acc = fmaf(S.yq[i * SY + q], Ef[c * W + q], acc);
            U[idx] = acc;
          }
          __syncthreads();
          cta_canon(U, mi, mi, r, sgn);
          for (int idx = tid; idx < mi * r; idx += BT) cp[idx] = U[idx];
          for (long long j = tid; j < cols; j += BT) {
            float b[W];
#pragma unroll
            for (int q = 0; q < W; ++q) b[q] = q < ks ? Bg[j * ks + q] : 0.f;
            for (int c = 0; c < r; ++c) {
              const float4* e4 = reinterpret_cast<const float4*>(Ef + c * W);
              float acc = 0.f;
#pragma unroll
              for (int q4 = 0; q4 < W / 4; ++q4) {
                const float4 e = e4[q4];
                if (4 * q4 + 0 < ks) acc = fmaf(b[4 * q4 + 0], e.x, acc);
                if (4 * q4 + 1 < ks) acc = fmaf(b[4 * q4 + 1], e.y, acc);
                if (4 * q4 + 2 < ks) acc = fmaf(b[4 * q4 + 2], e.z, acc);
                if (4 * q4 + 3 < ks) acc = fmaf(b[4 * q4 + 3], e.w, acc);
              }
              dst[j * r + c] = sgn[c] * acc;
            }
          }
        });
      } else {
        fail = true;
        if (tid == 0 && st) dev_fail(st, TT_ERR_UNSUPPORTED, t);
        break;
      }
      __syncthreads();
      cp += m * r;
      src = dst;
      size = (long long)r * cols;
      r_prev = r;
      if (tid == 0) ranks_out[(long long)t * (BMAXD + 1) + k + 1] = r;
    }
    if (!fail) {
      // last core = the remaining data (r_{d-1}, n_d, 1)
      for (long long i = tid; i < size; i += BT) cp[i] = src[i];
      if (tid == 0) {
        ranks_out[(long long)t * (BMAXD + 1) + d] = 1;
        err_out[t] = xn2 > 0.0 ? sqrt(tails / xn2) : 0.0;
      }
    }
    __syncthreads();
  }
}

// Shape table of a batch: validation and the per-CTA scratch the kernel needs.
struct BatchLayout {
  std::vector<BatchShape> hs;
  long long half = 0, per_cta = 0;
};

int batch_layout(int count, int d, const int* n, const long long* x_off, const long long* core_off, int rmax,
                 BatchLayout& L) {
  L.hs.assign((size_t)count, BatchShape{});
  long long maxsize = 0, maxbg = 0;
  for (int t = 0; t < count; ++t) {
    BatchShape& b = L.hs[(size_t)t];
    b.d = d;
    b.size = 1;
    for (int k = 0; k < BMAXD; ++k) b.n[k] = k < d ? n[(size_t)t * d + k] : 1;
    for (int k = 0; k < d; ++k) {
      if (b.n[k] < 1) {
        set_error(TT_ERR_SHAPE, "batched: tensor %d mode %d size %d", t, k, b.n[k]);
        return TT_ERR_SHAPE;
      }
      b.size *= b.n[k];
    }
    b.x_off = x_off[t];
    b.core_off = core_off[t];
    maxsize = std::max(maxsize, b.size);
    // randomized steps keep B (ks x cols) and need rows <= BMAXM
    long long rp = 1, sz = b.size;
    for (int k = 0; k < d - 1; ++k) {
      const long long m = rp * b.n[k], cols = sz / m, small = std::min(m, cols);
      if (small > BSMALL) {
        if (m > BMAXM) {
          set_error(TT_ERR_UNSUPPORTED, "batched: tensor %d step %d has %lld rows (> %d) on a sketched step", t, k, m,
                    BMAXM);
          return TT_ERR_UNSUPPORTED;
        }
        maxbg = std::max(maxbg, (long long)BSMALL * cols);
      }
      const long long rn = std::min<long long>((long long)rmax, small);
      sz = rn * cols;
      rp = rn;
    }
  }
  L.half = (maxsize + 63) & ~63LL;
  L.per_cta = 2 * L.half + ((maxbg + 63) & ~63LL);
  return TT_OK;
}

int check_batch_args(int count, int d, int rmax, double eps, int oversample) {
  if (count < 0 || d < 2 || d > BMAXD || rmax < 1 || rmax > BSMALL || !(eps >= 0.0) || oversample < 0) {
    set_error(TT_ERR_SHAPE, "batched: count %d, order %d (2..%d), rmax %d (1..%d), eps %g, oversample %d", count, d,
              BMAXD, rmax, BSMALL, eps, oversample);
    return TT_ERR_SHAPE;
  }
  return TT_OK;
}

template <int BCH>
int set_smem_attr() {
  return smem_optin_k(k_tt_batched<BCH>, sm_total<BCH>());
}

struct BatchArgs {
  const BatchShape* shp;
  const int* order;
  int count;
  const float* x;
  float* cores;
  int* ranks;
  double* err;
  float* scratch;
  long long per_cta, half;
  double eps;
  int rmax, oversample;
  unsigned long long seed;
  int* counter;
  DevStatus* st;
};

template <int BCH>
int launch_bch(int grid, cudaStream_t s, const BatchArgs& a) {
  TT_TRY(set_smem_attr<BCH>());
  k_tt_batched<BCH><<<grid, BT, sm_total<BCH>(), s>>>(a.shp, a.order, a.count, a.x, a.cores, a.ranks, a.err,
                                                       a.scratch, a.per_cta, a.half, a.eps, a.rmax, a.oversample,
                                                       a.seed, 40, a.counter, a.st);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

int launch_batched(int bch, int grid, cudaStream_t s, const BatchArgs& a) {
  switch (bch) {
    case 16: return launch_bch<16>(grid, s, a);
    case 32: return launch_bch<32>(grid, s, a);
    case 64: return launch_bch<64>(grid, s, a);
    default:
      set_error(TT_ERR_ARG, "batched: chunk width %d", bch);
      return TT_ERR_ARG;
  }
}

int persistent_grid(int count) { return std::max(1, std::min(count, dev_sms())); }

}  // namespace
}  // namespace ttr

using namespace ttr;

extern "C" long long tt_batch_core_capacity(int d, const int* n, int rmax) {
  if (d < 2 || d > BMAXD || !n || rmax < 1) return -1;
  long long total = 0, left = 1, right = 1;
  for (int k = 0; k < d; ++k) right *= n[k];
  long long rp = 1;
  for (int k = 0; k < d; ++k) {
    left *= n[k];
    right /= n[k];
    const long long rn = (k == d - 1) ? 1 : std::min<long long>({(long long)rmax, left, right});
    total += rp * n[k] * rn;
    rp = rn;
  }
  return total;
}

extern "C" int tt_svd_batched(tt_ctx* ctx, int count, int d, const int* n, const float* x,
                              const long long* x_off, double eps, int rmax, int oversample,
                              unsigned long long seed, float* cores, const long long* core_off, int* ranks,
                              double* err_est) {
  if (!ctx || !n || !x || !x_off || !cores || !core_off || !ranks || count < 0) {
    set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  TT_TRY(check_batch_args(count, d, rmax, eps, oversample));
  if (count == 0) return TT_OK;
  BatchLayout L;
  TT_TRY(batch_layout(count, d, n, x_off, core_off, rmax, L));
  const int grid = persistent_grid(count);
  const size_t bytes = sizeof(BatchShape) * (size_t)count + sizeof(int) * (size_t)count * (BMAXD + 1) +
                       sizeof(double) * (size_t)count + sizeof(float) * (size_t)L.per_cta * grid + 4096;
  Arena ws;
  TT_TRY(ctx_arena(ctx, bytes, &ws));
  BatchShape* dshp = ws.take<BatchShape>((size_t)count);
  int* dranks = ws.take<int>((size_t)count * (BMAXD + 1));
  double* derr = ws.take<double>((size_t)count);
  int* dcounter = ws.take<int>(1);
  float* scratch = ws.take<float>((size_t)L.per_cta * grid);
  if (!dshp || !dranks || !derr || !dcounter || !scratch) {
    set_error(TT_ERR_NOMEM, "batched workspace");
    return TT_ERR_NOMEM;
  }
  cudaStream_t s = ctx_stream(ctx);
  DevStatus* dst = ctx_status(ctx);
  TT_CUDA(cudaMemsetAsync(dst, 0, sizeof(DevStatus), s));
  TT_CUDA(cudaMemcpyAsync(dshp, L.hs.data(), sizeof(BatchShape) * (size_t)count, cudaMemcpyHostToDevice, s));
  TT_CUDA(cudaMemsetAsync(dcounter, 0, sizeof(int), s));
  const BatchArgs args{dshp, nullptr, count, x, cores, dranks, derr, scratch, L.per_cta, L.half,
                       eps, rmax, oversample, seed, dcounter, dst};
  TT_TRY(launch_batched(32, grid, s, args));
  std::vector<int> hr((size_t)count * (BMAXD + 1));
  TT_CUDA(cudaMemcpyAsync(hr.data(), dranks, sizeof(int) * hr.size(), cudaMemcpyDeviceToHost, s));
  if (err_est) TT_CUDA(cudaMemcpyAsync(err_est, derr, sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost, s));
  DevStatus hst;
  TT_CUDA(cudaMemcpyAsync(&hst, dst, sizeof(hst), cudaMemcpyDeviceToHost, s));
  TT_CUDA(cudaStreamSynchronize(s));
  for (int t = 0; t < count; ++t)
    for (int k = 0; k <= d; ++k) ranks[(size_t)t * (d + 1) + k] = hr[(size_t)t * (BMAXD + 1) + k];
  if (hst.code) {
    set_error(hst.code, "batched: device status %d (tensor %d)", hst.code, hst.detail);
    return hst.code;
  }
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// Batch plans: the batch's shape table, work orders and scratch allocated once, a variant
// (chunk width x work order) picked by timing every candidate on the batch, and the launch
// sequence (status reset, counter reset, persistent kernel, result read-back) captured in a
// CUDA graph that every later run replays with one cudaGraphLaunch.
// ---------------------------------------------------------------------------------------
struct tt_batch_plan {
  tt_ctx* ctx = nullptr;
  int count = 0, d = 0, rmax = 0, oversample = 0, grid = 1;
  double eps = 0.0;
  unsigned long long seed = 0;
  long long per_cta = 0, half = 0;
  char* dmem = nullptr;
  BatchShape* dshp = nullptr;
  int* dorder = nullptr;  // largest-first order
  int* dranks = nullptr;
  double* derr = nullptr;
  int* dcounter = nullptr;
  DevStatus* dst = nullptr;
  float* scratch = nullptr;
  int* hranks = nullptr;  // pinned
  double* herr = nullptr;
  DevStatus* hst = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, e0 = nullptr, e1 = nullptr;
  int bch = 32, sched = SCHED_LARGEST_FIRST;
  float tune_ms[6] = {0, 0, 0, 0, 0, 0};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const float* gx = nullptr;
  float* gcores = nullptr;
  int gbch = 0, gsched = -1;
};

namespace {
BatchArgs plan_args(tt_batch_plan* p, const float* x, float* cores, int sched) {
  return BatchArgs{p->dshp, sched == SCHED_LARGEST_FIRST ? p->dorder : nullptr, p->count, x, cores, p->dranks,
                   p->derr, p->scratch, p->per_cta, p->half, p->eps, p->rmax, p->oversample, p->seed, p->dcounter,
                   p->dst};
}

// The launch sequence of one run, on the plan's stream (also what the graph records).
int plan_enqueue(tt_batch_plan* p, const float* x, float* cores, int bch, int sched, bool readback) {
  cudaStream_t s = p->stream;
  TT_CUDA(cudaMemsetAsync(p->dst, 0, sizeof(DevStatus), s));
  TT_CUDA(cudaMemsetAsync(p->dcounter, 0, sizeof(int), s));
  TT_TRY(launch_batched(bch, p->grid, s, plan_args(p, x, cores, sched)));
  if (readback) {
    TT_CUDA(cudaMemcpyAsync(p->hranks, p->dranks, sizeof(int) * (size_t)p->count * (BMAXD + 1),
                            cudaMemcpyDeviceToHost, s));
    TT_CUDA(cudaMemcpyAsync(p->herr, p->derr, sizeof(double) * (size_t)p->count, cudaMemcpyDeviceToHost, s));
    TT_CUDA(cudaMemcpyAsync(p->hst, p->dst, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
  }
  return TT_OK;
}

void plan_drop_graph(tt_batch_plan* p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
  p->gx = nullptr;
  p->gcores = nullptr;
  p->gsched = -1;
}

int plan_capture(tt_batch_plan* p, const float* x, float* cores) {
  plan_drop_graph(p);
  TT_TRY(set_smem_attr<16>());
  TT_TRY(set_smem_attr<32>());
  TT_TRY(set_smem_attr<64>());
  TT_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = plan_enqueue(p, x, cores, p->bch, p->sched, true);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(p->stream, &g);
  if (rc != TT_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ec != cudaSuccess || !g) {
    set_error(TT_ERR_CUDA, "batched: graph capture: %s", cudaGetErrorString(ec));
    return TT_ERR_CUDA;
  }
  p->graph = g;
  if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) {
    p->exec = nullptr;
    plan_drop_graph(p);
    set_error(TT_ERR_CUDA, "batched: graph instantiation");
    return TT_ERR_CUDA;
  }
  p->gx = x;
  p->gcores = cores;
  p->gbch = p->bch;
  p->gsched = p->sched;
  return TT_OK;
}
}  // namespace

extern "C" int tt_batch_plan_destroy(tt_batch_plan* p) {
  if (!p) return TT_OK;
  if (p->stream) cudaStreamSynchronize(p->stream);
  plan_drop_graph(p);
  if (p->dmem) cudaFree(p->dmem);
  if (p->hranks) cudaFreeHost(p->hranks);
  if (p->herr) cudaFreeHost(p->herr);
  if (p->hst) cudaFreeHost(p->hst);
  if (p->ev_in) cudaEventDestroy(p->ev_in);
  if (p->e0) cudaEventDestroy(p->e0);
  if (p->e1) cudaEventDestroy(p->e1);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return TT_OK;
}

extern "C" int tt_batch_plan_create(tt_ctx* ctx, int count, int d, const int* n, const long long* x_off, double eps,
                                    int rmax, int oversample, unsigned long long seed, const long long* core_off,
                                    tt_batch_plan** out) {
  if (!ctx || !n || !x_off || !core_off || !out || count < 1) {
    set_error(TT_ERR_ARG, "batch plan: null argument or empty batch");
    return TT_ERR_ARG;
  }
  *out = nullptr;
  TT_TRY(check_batch_args(count, d, rmax, eps, oversample));
  BatchLayout L;
  TT_TRY(batch_layout(count, d, n, x_off, core_off, rmax, L));
  tt_batch_plan* p = new tt_batch_plan();
  p->ctx = ctx;
  p->count = count;
  p->d = d;
  p->rmax = rmax;
  p->oversample = oversample;
  p->eps = eps;
  p->seed = seed;
  p->per_cta = L.per_cta;
  p->half = L.half;
  p->grid = persistent_grid(count);
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_shp = carve(sizeof(BatchShape) * (size_t)count);
  const size_t o_ord = carve(sizeof(int) * (size_t)count);
  const size_t o_rk = carve(sizeof(int) * (size_t)count * (BMAXD + 1));
  const size_t o_err = carve(sizeof(double) * (size_t)count);
  const size_t o_cnt = carve(sizeof(int));
  const size_t o_st = carve(sizeof(DevStatus));
  const size_t o_scr = carve(sizeof(float) * (size_t)L.per_cta * p->grid);
  if (cudaMalloc(&p->dmem, off) != cudaSuccess ||
      cudaMallocHost(&p->hranks, sizeof(int) * (size_t)count * (BMAXD + 1)) != cudaSuccess ||
      cudaMallocHost(&p->herr, sizeof(double) * (size_t)count) != cudaSuccess ||
      cudaMallocHost(&p->hst, sizeof(DevStatus)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&p->e0) != cudaSuccess || cudaEventCreate(&p->e1) != cudaSuccess) {
    tt_batch_plan_destroy(p);
    set_error(TT_ERR_NOMEM, "batch plan allocation");
    return TT_ERR_NOMEM;
  }
  p->dshp = reinterpret_cast<BatchShape*>(p->dmem + o_shp);
  p->dorder = reinterpret_cast<int*>(p->dmem + o_ord);
  p->dranks = reinterpret_cast<int*>(p->dmem + o_rk);
  p->derr = reinterpret_cast<double*>(p->dmem + o_err);
  p->dcounter = reinterpret_cast<int*>(p->dmem + o_cnt);
  p->dst = reinterpret_cast<DevStatus*>(p->dmem + o_st);
  p->scratch = reinterpret_cast<float*>(p->dmem + o_scr);
  // largest-first order: the longest tensors start first, so the work counter's tail holds
  // only small ones (longest-processing-time rule for the SM makespan)
  std::vector<int> ord((size_t)count);
  for (int t = 0; t < count; ++t) ord[(size_t)t] = t;
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return L.hs[(size_t)a].size > L.hs[(size_t)b].size; });
  if (cudaMemcpyAsync(p->dshp, L.hs.data(), sizeof(BatchShape) * (size_t)count, cudaMemcpyHostToDevice, p->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(p->dorder, ord.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice, p->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(p->stream) != cudaSuccess) {
    tt_batch_plan_destroy(p);
    set_error(TT_ERR_CUDA, "batch plan upload");
    return TT_ERR_CUDA;
  }
  *out = p;
  return TT_OK;
}

extern "C" int tt_batch_plan_tune(tt_batch_plan* p, const float* x, float* cores, int reps, float* ms_out) {
  if (!p || !x || !cores) {
    set_error(TT_ERR_ARG, "batch plan tune: null argument");
    return TT_ERR_ARG;
  }
  reps = std::max(1, reps);
  TT_CUDA(cudaEventRecord(p->ev_in, ctx_stream(p->ctx)));
  TT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  float best = 0.f;
  int vi = 0;
  for (int sched = 0; sched < 2; ++sched)
    for (int c = 0; c < 3; ++c, ++vi) {
      TT_TRY(plan_enqueue(p, x, cores, kChunks[c], sched, false));  // warm-up
      TT_CUDA(cudaEventRecord(p->e0, p->stream));
      for (int r = 0; r < reps; ++r) TT_TRY(plan_enqueue(p, x, cores, kChunks[c], sched, false));
      TT_CUDA(cudaEventRecord(p->e1, p->stream));
      TT_CUDA(cudaEventSynchronize(p->e1));
      float ms = 0.f;
      TT_CUDA(cudaEventElapsedTime(&ms, p->e0, p->e1));
      ms /= (float)reps;
      p->tune_ms[vi] = ms;
      if (vi == 0 || ms < best) {
        best = ms;
        p->bch = kChunks[c];
        p->sched = sched;
      }
    }
  DevStatus h;
  TT_CUDA(cudaMemcpyAsync(&h, p->dst, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
  TT_CUDA(cudaStreamSynchronize(p->stream));
  if (h.code) {
    set_error(h.code, "batched: device status %d (tensor %d)", h.code, h.detail);
    return h.code;
  }
  if (ms_out)
    for (int i = 0; i < 6; ++i) ms_out[i] = p->tune_ms[i];
  return TT_OK;
}

extern "C" int tt_batch_plan_variant(const tt_batch_plan* p, int* chunk, int* largest_first) {
  if (!p) {
    set_error(TT_ERR_ARG, "batch plan: null");
    return TT_ERR_ARG;
  }
  if (chunk) *chunk = p->bch;
  if (largest_first) *largest_first = p->sched == SCHED_LARGEST_FIRST;
  return TT_OK;
}

extern "C" int tt_batch_plan_run(tt_batch_plan* p, const float* x, float* cores, int* ranks, double* err_est) {
  if (!p || !x || !cores) {
    set_error(TT_ERR_ARG, "batch plan run: null argument");
    return TT_ERR_ARG;
  }
  if (!p->exec || p->gx != x || p->gcores != cores || p->gbch != p->bch || p->gsched != p->sched)
    TT_TRY(plan_capture(p, x, cores));
  TT_CUDA(cudaEventRecord(p->ev_in, ctx_stream(p->ctx)));
  TT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  TT_CUDA(cudaGraphLaunch(p->exec, p->stream));
  count_launch();
  TT_CUDA(cudaStreamSynchronize(p->stream));
  if (ranks)
    for (int t = 0; t < p->count; ++t)
      for (int k = 0; k <= p->d; ++k)
        ranks[(size_t)t * (p->d + 1) + k] = p->hranks[(size_t)t * (BMAXD + 1) + k];
  if (err_est) memcpy(err_est, p->herr, sizeof(double) * (size_t)p->count);
  if (p->hst->code) {
    set_error(p->hst->code, "batched: device status %d (tensor %d)", p->hst->code, p->hst->detail);
    return p->hst->code;
  }
  return TT_OK;
}
