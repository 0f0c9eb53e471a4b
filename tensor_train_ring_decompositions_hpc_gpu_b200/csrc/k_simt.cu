// CUDA-core kernels: the plain-FP32 GEMM engine and every small linear-algebra kernel of the
// TT/TR-SVD chain (Gaussian test matrix, Gram matrices, CholeskyQR2, Jacobi eigen-solver,
// bond permute, core folding, reconstruction error).
#include <float.h>
#include <math.h>

#include <algorithm>

#include "kernels.cuh"

namespace ttr {

thread_local int g_kernel_launches = 0;

static int g_num_sms = 0;
static int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

// ---------------------------------------------------------------------------------------
// Philox4x32-10 Gaussian generator (replaces curandGenerateNormal, TT3O:585-587)
// ---------------------------------------------------------------------------------------
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

__global__ void k_gaussian(float* __restrict__ out, long long rows, long long total, long long ld,
                           unsigned long long seed, unsigned stream_id) {
  const long long ncall = (total + 3) / 4;
  const uint2 key = make_uint2((unsigned)(seed & 0xFFFFFFFFull), (unsigned)(seed >> 32));
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncall;
       c += (long long)gridDim.x * blockDim.x) {
    const uint4 w = philox4x32_10(
        make_uint4((unsigned)(c & 0xFFFFFFFFll), stream_id, (unsigned)(c >> 32), 0u), key);
    const float sc = 2.3283064365386963e-10f;  // 2^-32
    const float u0 = ((float)w.x + 0.5f) * sc, u1 = ((float)w.y + 0.5f) * sc;
    const float u2 = ((float)w.z + 0.5f) * sc, u3 = ((float)w.w + 0.5f) * sc;
    const float r0 = sqrtf(-2.0f * logf(u0)), r1 = sqrtf(-2.0f * logf(u2));
    float s0, c0, s1, c1;
    sincospif(2.0f * u1, &s0, &c0);
    sincospif(2.0f * u3, &s1, &c1);
    const float g[4] = {r0 * c0, r0 * s0, r1 * c1, r1 * s1};
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const long long e = 4 * c + l;
      if (e < total) {
        const long long row = e % rows, col = e / rows;
        out[row + ld * col] = g[l];
      }
    }
  }
}

int launch_gaussian(float* out, long long rows, int cols, long long ld, unsigned long long seed,
                    unsigned stream_id, cudaStream_t s) {
  const long long total = rows * (long long)cols;
  if (total <= 0) return TT_OK;
  const long long ncall = (total + 3) / 4;
  const int grid = (int)std::min<long long>(ceil_div_ll(ncall, 256), 8LL * num_sms());
  k_gaussian<<<grid, 256, 0, s>>>(out, rows, total, ld, seed, stream_id);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// Plain-FP32 sketch  Y = A * W  (split over the long dimension n, FP64 reduction of splits)
// ---------------------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(256) k_sketch_simt(const float* __restrict__ a, long long m,
                                                     long long n, const float* __restrict__ w,
                                                     int N, long long wj, long long wc,
                                                     long long jchunk, int cblk,
                                                     double* __restrict__ part) {
  constexpr int TI = 256, JC = 32, RI = 8, RC = NT / 8;
  __shared__ __align__(16) float as[JC][TI];
  __shared__ __align__(16) float wsm[JC][NT];
  const int tid = threadIdx.x;
  const long long i0 = (long long)blockIdx.x * TI;
  const int split = blockIdx.y;
  const int c0 = blockIdx.z * NT;
  const long long jb = (long long)split * jchunk;
  const long long je = (jb + jchunk < n) ? jb + jchunk : n;
  const int ti = tid >> 3, tc = tid & 7;
  float acc[RI][RC];
#pragma unroll
  for (int e = 0; e < RI; ++e)
#pragma unroll
    for (int c = 0; c < RC; ++c) acc[e][c] = 0.f;
  const bool vec = ((m & 3) == 0) && ((((uintptr_t)a) & 15) == 0);
  for (long long j0 = jb; j0 < je; j0 += JC) {
#pragma unroll
    for (int q = 0; q < (TI * JC / 4) / 256; ++q) {
      const int f = tid + 256 * q;
      const int jj = f / (TI / 4), i4 = f % (TI / 4);
      const long long j = j0 + jj, i = i0 + 4 * i4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j < je) {
        const float* p = a + j * m + i;
        if (vec && i + 3 < m) {
          v = __ldg(reinterpret_cast<const float4*>(p));
        } else {
          if (i < m) v.x = p[0];
          if (i + 1 < m) v.y = p[1];
          if (i + 2 < m) v.z = p[2];
          if (i + 3 < m) v.w = p[3];
        }
      }
      *reinterpret_cast<float4*>(&as[jj][4 * i4]) = v;
    }
    if (wc == 1) {
      for (int f = tid; f < JC * NT; f += 256) {
        const int c = f % NT, jj = f / NT;
        const long long j = j0 + jj;
        wsm[jj][c] = (j < je && c0 + c < N) ? w[j * wj + (long long)(c0 + c)] : 0.f;
      }
    } else {
      for (int f = tid; f < JC * NT; f += 256) {
        const int jj = f % JC, c = f / JC;
        const long long j = j0 + jj;
        wsm[jj][c] = (j < je && c0 + c < N) ? w[j * wj + (long long)(c0 + c) * wc] : 0.f;
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < JC; ++jj) {
      const float4 x0 = *reinterpret_cast<const float4*>(&as[jj][ti * RI]);
      const float4 x1 = *reinterpret_cast<const float4*>(&as[jj][ti * RI + 4]);
      const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      float wv[RC];
#pragma unroll
      for (int c = 0; c < RC; ++c) wv[c] = wsm[jj][tc * RC + c];
#pragma unroll
      for (int e = 0; e < RI; ++e)
#pragma unroll
        for (int c = 0; c < RC; ++c) acc[e][c] = fmaf(xv[e], wv[c], acc[e][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < RI; ++e) {
    const long long i = i0 + ti * RI + e;
#pragma unroll
    for (int c = 0; c < RC; ++c) {
      const int col = c0 + tc * RC + c;
      if (i < m && col < N) part[((long long)split * N + col) * m + i] = (double)acc[e][c];
    }
  }
  (void)cblk;
}

__global__ void k_reduce_splits(const double* __restrict__ part, long long count, int nsplit,
                                double* __restrict__ y) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < count;
       idx += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nsplit; ++k) s += part[(long long)k * count + idx];
    y[idx] = s;
  }
}

static void sketch_split_plan(long long m, long long n, long long* jchunk, int* nsplit) {
  const int mtiles = ceil_div(m, 256);
  const int target = 4 * num_sms();
  long long splits = std::max<long long>(1, target / std::max(1, mtiles));
  long long jc = ceil_div_ll(n, splits);
  if (jc < 256) jc = 256;
  jc = ceil_div_ll(jc, 32) * 32;
  *jchunk = jc;
  *nsplit = (int)ceil_div_ll(n, jc);
}

size_t sketch_ws_bytes(long long m, long long n, int N) {
  long long jchunk;
  int nsplit;
  sketch_split_plan(m, n, &jchunk, &nsplit);
  const size_t simt = (size_t)nsplit * (size_t)N * (size_t)m * sizeof(double) + 4096;
  return std::max(simt, sketch_tc_ws_bytes(m, n, N));
}

int launch_reduce_splits(const double* part, long long count, int nsplit, double* y, cudaStream_t s) {
  if (count <= 0) return TT_OK;
  k_reduce_splits<<<std::min(ceil_div(count, 256), 8 * num_sms()), 256, 0, s>>>(part, count, nsplit, y);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

int launch_sketch(const float* a, long long m, long long n, const float* w, int N, long long wj,
                  long long wc, double* y, int engine, Arena& ws, DevStatus* st, cudaStream_t s) {
  if (m <= 0 || n <= 0 || N <= 0) return TT_OK;
  if (engine == TT_GEMM_TC) {
    int rc = launch_sketch_tc(a, m, n, w, N, wj, wc, y, ws, st, s);
    if (rc != TT_ERR_UNSUPPORTED) return rc;
  }
  long long jchunk;
  int nsplit;
  sketch_split_plan(m, n, &jchunk, &nsplit);
  const size_t mk = ws.mark();
  double* part = ws.take<double>((size_t)nsplit * N * m);
  if (!part) {
    set_error(TT_ERR_NOMEM, "sketch workspace");
    return TT_ERR_NOMEM;
  }
  const int NT = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  const int cblk = ceil_div(N, NT);
  dim3 grid(ceil_div(m, 256), nsplit, cblk);
  switch (NT) {
    case 16: k_sketch_simt<16><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    case 32: k_sketch_simt<32><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    case 48: k_sketch_simt<48><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    default: k_sketch_simt<64><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
  }
  count_launch();
  TT_LAUNCH_CHECK();
  TT_TRY(launch_reduce_splits(part, (long long)N * m, nsplit, y, s));
  ws.reset(mk);
  return TT_OK;
}

// FP32 sketch with the split partials in caller-provided scratch (`part`, `part_cap` doubles);
// the split count is lowered until the partials fit.  Allocates nothing.
int launch_sketch_simt_static(const float* a, long long m, long long n, const float* w, int N,
                              long long wj, long long wc, double* y, double* part, size_t part_cap,
                              cudaStream_t s) {
  if (m <= 0 || n <= 0 || N <= 0) return TT_OK;
  long long jchunk;
  int nsplit;
  sketch_split_plan(m, n, &jchunk, &nsplit);
  const long long max_ns = (long long)(part_cap / ((size_t)N * (size_t)m));
  if (max_ns < 1) {
    set_error(TT_ERR_SHAPE, "sketch partials of %lld x %d doubles exceed the scratch of %zu doubles", m, N,
              part_cap);
    return TT_ERR_SHAPE;
  }
  if (nsplit > max_ns) {
    jchunk = (n + max_ns - 1) / max_ns;
    jchunk = (jchunk + 31) / 32 * 32;
    nsplit = (int)((n + jchunk - 1) / jchunk);
  }
  const int NT = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  const int cblk = ceil_div(N, NT);
  dim3 grid(ceil_div(m, 256), nsplit, cblk);
  switch (NT) {
    case 16: k_sketch_simt<16><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    case 32: k_sketch_simt<32><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    case 48: k_sketch_simt<48><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
    default: k_sketch_simt<64><<<grid, 256, 0, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
  }
  count_launch();
  TT_LAUNCH_CHECK();
  return launch_reduce_splits(part, (long long)N * m, nsplit, y, s);
}

// ---------------------------------------------------------------------------------------
// Plain-FP32 projection  out = A^T Q  (A column-major m x n, contraction over m)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int swz(int row, int col) { return col ^ (((row >> 2) & 7) << 2); }

template <int NT>
__global__ void __launch_bounds__(256) k_project_simt(const float* __restrict__ a, long long m,
                                                      long long n, const float* __restrict__ q,
                                                      int N, long long ldq, float* __restrict__ out,
                                                      long long ldo, int mode, int r0, int r1) {
  constexpr int TJ = 256, KC = 32, RJ = 8, RC = NT / 8;
  __shared__ __align__(16) float as[KC][TJ];
  __shared__ __align__(16) float qs[KC][NT];
  const int tid = threadIdx.x;
  const long long j0 = (long long)blockIdx.x * TJ;
  const int c0 = blockIdx.y * NT;
  const int tj = tid >> 3, tc = tid & 7;
  float acc[RJ][RC];
#pragma unroll
  for (int e = 0; e < RJ; ++e)
#pragma unroll
    for (int c = 0; c < RC; ++c) acc[e][c] = 0.f;
  const bool vec = ((m & 3) == 0) && ((((uintptr_t)a) & 15) == 0);
  for (long long k0 = 0; k0 < m; k0 += KC) {
#pragma unroll
    for (int qq = 0; qq < (TJ * KC / 4) / 256; ++qq) {
      const int f = tid + 256 * qq;
      const int jj = f >> 3, k4 = f & 7;
      const long long j = j0 + jj, k = k0 + 4 * k4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j < n) {
        const float* p = a + j * m + k;
        if (vec && k + 3 < m) {
          v = __ldg(reinterpret_cast<const float4*>(p));
        } else {
          if (k < m) v.x = p[0];
          if (k + 1 < m) v.y = p[1];
          if (k + 2 < m) v.z = p[2];
          if (k + 3 < m) v.w = p[3];
        }
      }
      const int kk = 4 * k4;
      as[kk + 0][swz(kk + 0, jj)] = v.x;
      as[kk + 1][swz(kk + 1, jj)] = v.y;
      as[kk + 2][swz(kk + 2, jj)] = v.z;
      as[kk + 3][swz(kk + 3, jj)] = v.w;
    }
    for (int f = tid; f < KC * NT; f += 256) {
      const int kk = f % KC, c = f / KC;
      const long long k = k0 + kk;
      qs[kk][c] = (k < m && c0 + c < N) ? q[k + ldq * (long long)(c0 + c)] : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KC; ++kk) {
      const float4 x0 = *reinterpret_cast<const float4*>(&as[kk][swz(kk, tj * RJ)]);
      const float4 x1 = *reinterpret_cast<const float4*>(&as[kk][swz(kk, tj * RJ + 4)]);
      const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      float qv[RC];
#pragma unroll
      for (int c = 0; c < RC; ++c) qv[c] = qs[kk][tc * RC + c];
#pragma unroll
      for (int e = 0; e < RJ; ++e)
#pragma unroll
        for (int c = 0; c < RC; ++c) acc[e][c] = fmaf(xv[e], qv[c], acc[e][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < RJ; ++e) {
    const long long j = j0 + tj * RJ + e;
    if (j >= n) continue;
#pragma unroll
    for (int c = 0; c < RC; ++c) {
      const int col = c0 + tc * RC + c;
      if (col >= N) continue;
      if (mode == OUT_ROWMAJOR) {
        out[j * ldo + col] = acc[e][c];
      } else {
        const int ai = col % r0, bi = col / r0;
        out[(long long)bi + (long long)r1 * (j + n * (long long)ai)] = acc[e][c];
      }
    }
  }
}

int launch_project(const float* a, long long m, long long n, const float* q, int N, long long ldq,
                   float* out, long long ldo, int mode, int r0, int r1, int engine, Arena& ws,
                   DevStatus* st, cudaStream_t s) {
  if (n <= 0 || N <= 0) return TT_OK;
  if (engine == TT_GEMM_TC) {
    int rc = launch_project_tc(a, m, n, q, N, ldq, out, ldo, mode, r0, r1, ws, st, s);
    if (rc != TT_ERR_UNSUPPORTED) return rc;
  }
  const int NT = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  dim3 grid(ceil_div(n, 256), ceil_div(N, NT));
  switch (NT) {
    case 16: k_project_simt<16><<<grid, 256, 0, s>>>(a, m, n, q, N, ldq, out, ldo, mode, r0, r1); break;
    case 32: k_project_simt<32><<<grid, 256, 0, s>>>(a, m, n, q, N, ldq, out, ldo, mode, r0, r1); break;
    case 48: k_project_simt<48><<<grid, 256, 0, s>>>(a, m, n, q, N, ldq, out, ldo, mode, r0, r1); break;
    default: k_project_simt<64><<<grid, 256, 0, s>>>(a, m, n, q, N, ldq, out, ldo, mode, r0, r1); break;
  }
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// Gram  W = sum_j x_j x_j^T  (M <= 128), symmetric 4x4 register tiles, FP64 across blocks
// ---------------------------------------------------------------------------------------
template <int MP, bool ACC64>
__global__ void __launch_bounds__(256) k_gram(const float* __restrict__ x, long long nvec, int M,
                                              long long vs, long long es, long long vchunk,
                                              double* __restrict__ part) {
  constexpr int VC = 32;
  constexpr int TT = MP / 4;
  constexpr int NTILE = TT * (TT + 1) / 2;
  constexpr int GROUPS = NTILE >= 256 ? 1 : 256 / NTILE;
  constexpr int TPT = NTILE >= 256 ? (NTILE + 255) / 256 : 1;
  __shared__ __align__(16) float xs[VC][MP];
  __shared__ double red[GROUPS > 1 ? MP * MP : 1];
  const int tid = threadIdx.x;
  const long long vb = (long long)blockIdx.x * vchunk;
  const long long ve = (vb + vchunk < nvec) ? vb + vchunk : nvec;

  int ta[TPT], tb[TPT];
  bool act[TPT];
  int g = 0;
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    int t = (GROUPS > 1) ? (tid % NTILE) : (tid + 256 * u);
    if (GROUPS > 1) g = tid / NTILE;
    act[u] = (GROUPS > 1) ? (g < GROUPS) : (t < NTILE);
    int aa = 0, rem = act[u] ? t : 0;
    while (rem >= TT - aa) {
      rem -= TT - aa;
      ++aa;
    }
    ta[u] = aa;
    tb[u] = aa + rem;
  }
  float acc[TPT][16];
  double accd[TPT][16];
#pragma unroll
  for (int u = 0; u < TPT; ++u)
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      acc[u][e] = 0.f;
      accd[u][e] = 0.0;
    }
  int chunk = 0;
  for (long long v0 = vb; v0 < ve; v0 += VC, ++chunk) {
    if (es == 1) {
      for (int f = tid; f < VC * MP; f += 256) {
        const int c = f % MP, v = f / MP;
        const long long j = v0 + v;
        xs[v][c] = (j < ve && c < M) ? x[j * vs + c] : 0.f;
      }
    } else {
      for (int f = tid; f < VC * MP; f += 256) {
        const int v = f % VC, c = f / VC;
        const long long j = v0 + v;
        xs[v][c] = (j < ve && c < M) ? x[j * vs + (long long)c * es] : 0.f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      if (!act[u]) continue;
      for (int v = g; v < VC; v += GROUPS) {
        const float4 xa = *reinterpret_cast<const float4*>(&xs[v][ta[u] * 4]);
        const float4 xb = *reinterpret_cast<const float4*>(&xs[v][tb[u] * 4]);
        const float av[4] = {xa.x, xa.y, xa.z, xa.w};
        const float bv[4] = {xb.x, xb.y, xb.z, xb.w};
        if (ACC64) {
#pragma unroll
          for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int r = 0; r < 4; ++r)
              accd[u][p * 4 + r] = fma((double)av[p], (double)bv[r], accd[u][p * 4 + r]);
        } else {
#pragma unroll
          for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[u][p * 4 + r] = fmaf(av[p], bv[r], acc[u][p * 4 + r]);
        }
      }
    }
    if (!ACC64 && (chunk & 31) == 31) {
#pragma unroll
      for (int u = 0; u < TPT; ++u)
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          accd[u][e] += (double)acc[u][e];
          acc[u][e] = 0.f;
        }
    }
    __syncthreads();
  }
  if (!ACC64) {
#pragma unroll
    for (int u = 0; u < TPT; ++u)
#pragma unroll
      for (int e = 0; e < 16; ++e) accd[u][e] += (double)acc[u][e];
  }
  double* dst = part + (long long)blockIdx.x * MP * MP;
  if (GROUPS > 1) {
    for (int gg = 0; gg < GROUPS; ++gg) {
      if (g == gg && act[0]) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int idx = (ta[0] * 4 + p) * MP + tb[0] * 4 + r;
            red[idx] = (gg == 0) ? accd[0][p * 4 + r] : red[idx] + accd[0][p * 4 + r];
          }
      }
      __syncthreads();
    }
    if (g == 0 && act[0]) {
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int idx = (ta[0] * 4 + p) * MP + tb[0] * 4 + r;
          dst[idx] = red[idx];
        }
    }
  } else {
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      if (!act[u]) continue;
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int r = 0; r < 4; ++r) dst[(ta[u] * 4 + p) * MP + tb[u] * 4 + r] = accd[u][p * 4 + r];
    }
  }
}

__global__ void k_gram_reduce(const double* __restrict__ part, int nblk, int MP, int M,
                              double* __restrict__ w) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M * M) return;
  const int aI = idx % M, bI = idx / M;
  const int src = (aI / 4 <= bI / 4) ? aI * MP + bI : bI * MP + aI;
  double sacc = 0.0;
  for (int k = 0; k < nblk; ++k) sacc += part[(long long)k * MP * MP + src];
  w[aI + (long long)M * bI] = sacc;
}

static int gram_mp(int M) { return M <= 16 ? 16 : M <= 32 ? 32 : M <= 48 ? 48 : M <= 64 ? 64 : 128; }

static void gram_plan(long long nvec, int* nblk, long long* vchunk) {
  const int target = 4 * num_sms();
  long long vc = ceil_div_ll(nvec, target);
  if (vc < 1024) vc = 1024;
  vc = ceil_div_ll(vc, 32) * 32;
  *vchunk = vc;
  *nblk = (int)std::max<long long>(1, ceil_div_ll(nvec, vc));
}

size_t gram_ws_bytes(long long nvec, int M) {
  int nblk;
  long long vc;
  gram_plan(nvec, &nblk, &vc);
  const int MP = gram_mp(M);
  return (size_t)nblk * MP * MP * sizeof(double) + 4096;
}

int launch_gram(const float* x, long long nvec, int M, long long vs, long long es, double* w,
                bool acc64, Arena& ws, cudaStream_t s) {
  if (M <= 0) return TT_OK;
  if (M > TT_MAX_SMALL) {
    set_error(TT_ERR_UNSUPPORTED, "gram size %d > %d", M, TT_MAX_SMALL);
    return TT_ERR_UNSUPPORTED;
  }
  int nblk;
  long long vchunk;
  gram_plan(std::max<long long>(nvec, 1), &nblk, &vchunk);
  const int MP = gram_mp(M);
  const size_t mk = ws.mark();
  double* part = ws.take<double>((size_t)nblk * MP * MP);
  if (!part) {
    set_error(TT_ERR_NOMEM, "gram workspace");
    return TT_ERR_NOMEM;
  }
#define GRAM_CASE(MPV)                                                                      \
  case MPV:                                                                                 \
    if (acc64)                                                                              \
      k_gram<MPV, true><<<nblk, 256, 0, s>>>(x, nvec, M, vs, es, vchunk, part);             \
    else                                                                                    \
      k_gram<MPV, false><<<nblk, 256, 0, s>>>(x, nvec, M, vs, es, vchunk, part);            \
    break;
  switch (MP) {
    GRAM_CASE(16)
    GRAM_CASE(32)
    GRAM_CASE(48)
    GRAM_CASE(64)
    GRAM_CASE(128)
  }
#undef GRAM_CASE
  count_launch();
  TT_LAUNCH_CHECK();
  k_gram_reduce<<<ceil_div(M * M, 256), 256, 0, s>>>(part, nblk, MP, M, w);
  count_launch();
  TT_LAUNCH_CHECK();
  ws.reset(mk);
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// CholeskyQR2: FP64 Cholesky + triangular inverse on chip, FP32 apply
// ---------------------------------------------------------------------------------------
// One block: W (N x N, FP64) -> R (upper, FP64) and R^-1 (FP64).  Pivots below
// rel_tol * max diag mark a dependent column: its row of R and column of R^-1 are zero.
__global__ void __launch_bounds__(256) k_chol_inv(const double* __restrict__ w, int N,
                                                  double* __restrict__ r_out,
                                                  double* __restrict__ rinv, double rel_tol,
                                                  DevStatus* st) {
  extern __shared__ double sm[];
  double* A = sm;                 // N x N (row-major), upper part becomes R
  int* dead = reinterpret_cast<int*>(sm + N * N);
  __shared__ double piv_s, dmax_s;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < N * N; idx += blockDim.x) {
    const int i = idx / N, j = idx % N;
    A[idx] = w[i + (long long)N * j];
  }
  if (tid == 0) {
    double dm = 0.0;
    for (int i = 0; i < N; ++i) dm = fmax(dm, w[i + (long long)N * i]);
    dmax_s = dm;
  }
  __syncthreads();
  const double tol = rel_tol * dmax_s;
  for (int k = 0; k < N; ++k) {
    if (tid == 0) {
      const double d = A[k * N + k];
      if (!(d > tol) || dmax_s <= 0.0) {
        dead[k] = 1;
        piv_s = 0.0;
      } else {
        dead[k] = 0;
        piv_s = sqrt(d);
      }
    }
    __syncthreads();
    const double pv = piv_s;
    for (int j = k + tid; j < N; j += blockDim.x) {
      if (pv == 0.0) {
        A[k * N + j] = 0.0;
      } else {
        A[k * N + j] = (j == k) ? pv : A[k * N + j] / pv;
      }
    }
    __syncthreads();
    const int rem = N - k - 1;
    for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
      const int i = k + 1 + idx / rem, j = k + 1 + idx % rem;
      if (j >= i) A[i * N + j] -= A[k * N + i] * A[k * N + j];
    }
    __syncthreads();
  }
  // R out (column-major), zero below the diagonal; dead diagonal entries stay 0.
  if (r_out) {
    for (int idx = tid; idx < N * N; idx += blockDim.x) {
      const int i = idx % N, j = idx / N;
      r_out[idx] = (j >= i) ? A[i * N + j] : 0.0;
    }
  }
  // R^-1 column by column (column-major output in global memory).
  for (int idx = tid; idx < N * N; idx += blockDim.x) rinv[idx] = 0.0;
  __syncthreads();
  for (int j = 0; j < N; ++j) {
    if (dead[j]) continue;  // uniform across the block
    const double rjj = A[j * N + j];
    for (int i = tid; i <= j; i += blockDim.x) {
      double v;
      if (i == j) {
        v = 1.0 / rjj;
      } else if (dead[i]) {
        v = 0.0;
      } else {
        double acc = 0.0;
        for (int k = i; k < j; ++k) acc += rinv[i + (long long)N * k] * A[k * N + j];
        v = -acc / rjj;
      }
      rinv[i + (long long)N * j] = v;
    }
    __syncthreads();
  }
  (void)st;
}

// Y (n x N) <- Y * T, T = R^-1 upper (FP64 in global, staged as FP32).  128 rows per block,
// one row per thread, outputs produced 32 columns at a time.
template <int NP>
__global__ void __launch_bounds__(128) k_apply_rinv(float* __restrict__ y, long long n, int N,
                                                    long long vs, long long es,
                                                    const double* __restrict__ t) {
  extern __shared__ float sm_apply[];
  float* ts = sm_apply;                 // NP x NP, ts[k*NP + c]
  float* ys = ts + NP * NP;             // 128 x (NP+1)
  float* yo = ys + 128 * (NP + 1);      // 128 x (NP+1)
  constexpr int LD = NP + 1;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NP * NP; idx += 128) {
    const int k = idx % NP, c = idx / NP;
    ts[k * NP + c] = (k < N && c < N) ? (float)t[k + (long long)N * c] : 0.f;
  }
  const long long j0 = (long long)blockIdx.x * 128;
  if (es == 1) {
    for (int f = tid; f < 128 * NP; f += 128) {
      const int c = f % NP, r = f / NP;
      const long long j = j0 + r;
      ys[r * LD + c] = (j < n && c < N) ? y[j * vs + c] : 0.f;
    }
  } else {
    for (int f = tid; f < 128 * NP; f += 128) {
      const int r = f % 128, c = f / 128;
      const long long j = j0 + r;
      ys[r * LD + c] = (j < n && c < N) ? y[j * vs + (long long)c * es] : 0.f;
    }
  }
  __syncthreads();
  // Output chunk width divides NP (NP is a multiple of 16), so cb + c < NP always.
  constexpr int CB = (NP % 32 == 0) ? 32 : 16;
  static_assert(NP % CB == 0, "chunk width must divide the padded width");
  for (int cb = 0; cb < NP; cb += CB) {
    float outv[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) outv[c] = 0.f;
    for (int k = 0; k < cb + CB && k < NP; ++k) {
      const float yk = ys[tid * LD + k];
#pragma unroll
      for (int c = 0; c < CB; ++c) outv[c] = fmaf(yk, ts[k * NP + cb + c], outv[c]);
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) yo[tid * LD + cb + c] = outv[c];
  }
  __syncthreads();
  if (es == 1) {
    for (int f = tid; f < 128 * NP; f += 128) {
      const int c = f % NP, r = f / NP;
      const long long j = j0 + r;
      if (j < n && c < N) y[j * vs + c] = yo[r * LD + c];
    }
  } else {
    for (int f = tid; f < 128 * NP; f += 128) {
      const int r = f % 128, c = f / 128;
      const long long j = j0 + r;
      if (j < n && c < N) y[j * vs + (long long)c * es] = yo[r * LD + c];
    }
  }
}

// R = R2 * R1 (upper triangular, FP64).
__global__ void k_mul_upper(const double* __restrict__ r2, const double* __restrict__ r1, int N,
                            double* __restrict__ r) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * N) return;
  const int i = idx % N, j = idx / N;
  double acc = 0.0;
  for (int k = i; k <= j; ++k) acc += r2[i + (long long)N * k] * r1[k + (long long)N * j];
  r[idx] = (j >= i) ? acc : 0.0;
}

int launch_cholqr2(float* y, long long n, int N, long long vs, long long es, double* r,
                   Arena& ws, DevStatus* st, cudaStream_t s) {
  if (N <= 0 || n <= 0) return TT_OK;
  if (N > TT_MAX_SMALL) {
    set_error(TT_ERR_UNSUPPORTED, "cholqr2 width %d > %d", N, TT_MAX_SMALL);
    return TT_ERR_UNSUPPORTED;
  }
  const size_t mk = ws.mark();
  double* w = ws.take<double>((size_t)N * N);
  double* rinv = ws.take<double>((size_t)N * N);
  double* r1 = ws.take<double>((size_t)N * N);
  double* r2 = ws.take<double>((size_t)N * N);
  if (!w || !rinv || !r1 || !r2) {
    set_error(TT_ERR_NOMEM, "cholqr2 workspace");
    return TT_ERR_NOMEM;
  }
  const int NP = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : N <= 64 ? 64 : 128;
  const size_t shm = (size_t)N * N * sizeof(double) + N * sizeof(int) + 16;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_apply_rinv<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_apply_rinv<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_apply_rinv<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_apply_rinv<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_apply_rinv<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  for (int pass = 0; pass < 2; ++pass) {
    TT_TRY(launch_gram(y, n, N, vs, es, w, true, ws, s));
    k_chol_inv<<<1, 256, shm, s>>>(w, N, pass == 0 ? r1 : r2, rinv, 1e-12, st);
    count_launch();
    TT_LAUNCH_CHECK();
    const int grid = ceil_div(n, 128);
    const size_t ashm = ((size_t)NP * NP + 2 * 128 * (size_t)(NP + 1)) * sizeof(float);
    switch (NP) {
      case 16: k_apply_rinv<16><<<grid, 128, ashm, s>>>(y, n, N, vs, es, rinv); break;
      case 32: k_apply_rinv<32><<<grid, 128, ashm, s>>>(y, n, N, vs, es, rinv); break;
      case 48: k_apply_rinv<48><<<grid, 128, ashm, s>>>(y, n, N, vs, es, rinv); break;
      case 64: k_apply_rinv<64><<<grid, 128, ashm, s>>>(y, n, N, vs, es, rinv); break;
      default: k_apply_rinv<128><<<grid, 128, ashm, s>>>(y, n, N, vs, es, rinv); break;
    }
    count_launch();
    TT_LAUNCH_CHECK();
  }
  if (r) {
    k_mul_upper<<<ceil_div(N * N, 256), 256, 0, s>>>(r2, r1, N, r);
    count_launch();
    TT_LAUNCH_CHECK();
  }
  ws.reset(mk);
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// Symmetric eigen-decomposition: parallel cyclic Jacobi (round-robin pairs), FP64
// ---------------------------------------------------------------------------------------
// W is held row-major in shared memory, V in shared memory (N <= 64) or global memory.
template <bool VSMEM>
__global__ void __launch_bounds__(256) k_syev_jacobi(const double* __restrict__ w_in, int N,
                                                     double* __restrict__ evals,
                                                     double* __restrict__ evecs,
                                                     double* __restrict__ vglob, int max_sweeps,
                                                     DevStatus* st) {
  extern __shared__ double sm[];
  const int Np = N + (N & 1);
  double* W = sm;                             // Np x Np
  double* V = VSMEM ? sm + Np * Np : vglob;   // Np x Np
  double* cs = sm + (VSMEM ? 2 : 1) * Np * Np;
  double* sn = cs + Np / 2;
  int* pp = reinterpret_cast<int*>(sn + Np / 2);
  int* qq = pp + Np / 2;
  int* order = qq + Np / 2;
  __shared__ int nrot;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int idx = tid; idx < Np * Np; idx += nt) {
    const int i = idx / Np, j = idx % Np;
    W[idx] = (i < N && j < N) ? w_in[i + (long long)N * j] : 0.0;
    V[idx] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const double tol = 1e-14;
  int sweep = 0;
  bool converged = false;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) nrot = 0;
    __syncthreads();
    for (int rnd = 0; rnd < Np - 1; ++rnd) {
      for (int k = tid; k < Np / 2; k += nt) {
        const int x = k, y = Np - 1 - k;
        int p = (x == 0) ? 0 : 1 + (x - 1 + rnd) % (Np - 1);
        int q = (y == 0) ? 0 : 1 + (y - 1 + rnd) % (Np - 1);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, s = 0.0;
        if (q < N) {
          const double apq = W[p * Np + q], app = W[p * Np + p], aqq = W[q * Np + q];
          if (fabs(apq) > tol * sqrt(fabs(app * aqq)) && apq != 0.0) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(1.0 + theta * theta));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
            atomicAdd(&nrot, 1);
          }
        }
        cs[k] = c;
        sn[k] = s;
        pp[k] = p;
        qq[k] = q;
      }
      __syncthreads();
      // rows: W <- J^T W
      for (int idx = tid; idx < (Np / 2) * Np; idx += nt) {
        const int k = idx / Np, j = idx % Np;
        const double c = cs[k], s = sn[k];
        if (s == 0.0) continue;
        const int p = pp[k], q = qq[k];
        const double wp = W[p * Np + j], wq = W[q * Np + j];
        W[p * Np + j] = c * wp - s * wq;
        W[q * Np + j] = s * wp + c * wq;
      }
      __syncthreads();
      // columns: W <- W J, V <- V J
      for (int idx = tid; idx < (Np / 2) * Np; idx += nt) {
        const int k = idx / Np, i = idx % Np;
        const double c = cs[k], s = sn[k];
        if (s == 0.0) continue;
        const int p = pp[k], q = qq[k];
        const double wp = W[i * Np + p], wq = W[i * Np + q];
        W[i * Np + p] = c * wp - s * wq;
        W[i * Np + q] = s * wp + c * wq;
        const double vp = V[i * Np + p], vq = V[i * Np + q];
        V[i * Np + p] = c * vp - s * vq;
        V[i * Np + q] = s * vp + c * vq;
      }
      __syncthreads();
    }
    if (nrot == 0) {
      converged = true;
      break;
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int i = 0; i < N; ++i) order[i] = i;
    for (int i = 0; i < N; ++i) {  // selection sort, descending eigenvalues
      int best = i;
      for (int j = i + 1; j < N; ++j)
        if (W[order[j] * Np + order[j]] > W[order[best] * Np + order[best]]) best = j;
      const int t = order[i];
      order[i] = order[best];
      order[best] = t;
    }
    if (st) {
      atomicMax(&st->sweeps, sweep + 1);
      if (!converged) dev_fail(st, TT_ERR_NOCONV, sweep);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < N * N; idx += nt) {
    const int i = idx % N, a = idx / N;
    evecs[i + (long long)N * a] = V[i * Np + order[a]];
  }
  for (int a = tid; a < N; a += nt) evals[a] = W[order[a] * Np + order[a]];
}

int launch_syev(const double* w, int N, double* evals, double* evecs, int max_sweeps, Arena& ws,
                DevStatus* st, cudaStream_t s) {
  if (N <= 0) return TT_OK;
  if (N > TT_MAX_SMALL) {
    set_error(TT_ERR_UNSUPPORTED, "eigen-solver size %d > %d", N, TT_MAX_SMALL);
    return TT_ERR_UNSUPPORTED;
  }
  const int Np = N + (N & 1);
  const bool vsm = Np <= 64;
  const size_t shm = (size_t)(vsm ? 2 : 1) * Np * Np * sizeof(double) + Np * sizeof(double) +
                     (size_t)Np / 2 * 2 * sizeof(int) + Np * sizeof(int) + 64;
  const size_t mk = ws.mark();
  double* vg = nullptr;
  if (!vsm) {
    vg = ws.take<double>((size_t)Np * Np);
    if (!vg) {
      set_error(TT_ERR_NOMEM, "jacobi workspace");
      return TT_ERR_NOMEM;
    }
  }
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_syev_jacobi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_syev_jacobi<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  if (vsm)
    k_syev_jacobi<true><<<1, 256, shm, s>>>(w, N, evals, evecs, vg, max_sweeps, st);
  else
    k_syev_jacobi<false><<<1, 256, shm, s>>>(w, N, evals, evecs, vg, max_sweeps, st);
  count_launch();
  TT_LAUNCH_CHECK();
  ws.reset(mk);
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// TR bond permute (r0, r1, n) -> (r1, n, r0), staged through shared memory
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_permute231(const float* __restrict__ in,
                                                    float* __restrict__ out, int r0, int r1,
                                                    long long n, int jt) {
  extern __shared__ float tile[];  // jt * r0 * r1 floats
  const long long j0 = (long long)blockIdx.x * jt;
  const int q = r0 * r1;
  const long long jn = (j0 + jt <= n) ? jt : (n - j0);
  const long long cnt = jn * q;
  const float* src = in + j0 * q;
  for (long long f = threadIdx.x; f < cnt; f += blockDim.x) tile[f] = src[f];
  __syncthreads();
  // out[b + r1*(j + n*a)]: for each a, a contiguous run of r1*jn floats
  for (long long f = threadIdx.x; f < cnt; f += blockDim.x) {
    const int a = (int)(f / (r1 * jn));
    const long long rem = f % (r1 * jn);
    const int b = (int)(rem % r1);
    const long long jj = rem / r1;
    out[(long long)r1 * (j0 + n * a) + rem] = tile[jj * q + a + (long long)r0 * b];
  }
}

int launch_permute231(const float* in, float* out, int r0, int r1, long long n, cudaStream_t s) {
  const int q = r0 * r1;
  if (q <= 0 || n <= 0) return TT_OK;
  int jt = std::max(1, 8192 / q);
  const size_t shm = (size_t)jt * q * sizeof(float);
  k_permute231<<<(int)ceil_div_ll(n, jt), 256, shm, s>>>(in, out, r0, r1, n, jt);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------------------
__global__ void k_small_nn(const float* __restrict__ a, long long M, int K, long long lda,
                           const double* __restrict__ b, int N, long long ldb,
                           const double* __restrict__ colscale, int nvalid,
                           float* __restrict__ c, long long ldc) {
  const long long total = M * (long long)N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % M;
    const int col = (int)(idx / M);
    double acc = 0.0;
    if (col < nvalid) {
      for (int k = 0; k < K; ++k) acc += (double)a[i + lda * k] * b[k + ldb * col];
      if (colscale) acc *= colscale[col];
    }
    c[i + ldc * col] = (float)acc;
  }
}

int launch_small_nn(const float* a, long long M, int K, long long lda, const double* b, int N,
                    long long ldb, const double* colscale, int nvalid, float* c, long long ldc,
                    cudaStream_t s) {
  const long long total = M * (long long)N;
  if (total <= 0) return TT_OK;
  k_small_nn<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0, s>>>(
      a, M, K, lda, b, N, ldb, colscale, nvalid, c, ldc);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_fold_rows(const float* __restrict__ in, float* __restrict__ out,
                            const double* __restrict__ p, int R, long long ni, int ncols) {
  const long long M = (long long)R * ni;
  const long long total = M * ncols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long row = idx % M;
    const long long bcol = idx / M;
    const int a = (int)(row % R);
    const long long i = row / R;
    double acc = 0.0;
    for (int ap = 0; ap < R; ++ap)
      acc += p[ap + (long long)R * a] * (double)in[(ap + (long long)R * i) + M * bcol];
    out[idx] = (float)acc;
  }
}

int launch_fold_rows(const float* in, float* out, const double* p, int R, long long ni, int ncols,
                     cudaStream_t s) {
  const long long total = (long long)R * ni * ncols;
  if (total <= 0) return TT_OK;
  k_fold_rows<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0, s>>>(
      in, out, p, R, ni, ncols);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_f64_to_f32_cols(const double* __restrict__ in, long long rows, long long ldin,
                                  int k, float* __restrict__ out, long long ldout, int ncols) {
  const long long total = rows * ncols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % rows;
    const int c = (int)(idx / rows);
    out[i + ldout * c] = (c < k) ? (float)in[i + ldin * c] : 0.f;
  }
}

int launch_f64_to_f32_cols(const double* in, long long rows, long long ldin, int k, float* out,
                           long long ldout, int ncols, cudaStream_t s) {
  const long long total = rows * ncols;
  if (total <= 0) return TT_OK;
  k_f64_to_f32_cols<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0,
                      s>>>(in, rows, ldin, k, out, ldout, ncols);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_sigma_vt(const double* __restrict__ evals, const double* __restrict__ v, int n,
                           int k, int kvalid, float* __restrict__ out) {
  const int total = n * k;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int a = idx % k, j = idx / k;
    out[idx] = (a < kvalid) ? (float)(sqrt(fmax(evals[a], 0.0)) * v[j + (long long)n * a]) : 0.f;
  }
}

int launch_sigma_vt(const double* evals, const double* v, int n, int k, int kvalid, float* out,
                    cudaStream_t s) {
  if (n * k <= 0) return TT_OK;
  k_sigma_vt<<<ceil_div(n * k, 256), 256, 0, s>>>(evals, v, n, k, kvalid, out);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_inv_sigma(const double* __restrict__ evals, int k, double* __restrict__ cs,
                            double rel_floor) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= k) return;
  const double s0 = sqrt(fmax(evals[0], 0.0));
  const double sa = sqrt(fmax(evals[a], 0.0));
  cs[a] = (sa > rel_floor * s0 && sa > 0.0) ? 1.0 / sa : 0.0;
}

int launch_inv_sigma(const double* evals, int k, double* colscale, double rel_floor, cudaStream_t s) {
  if (k <= 0) return TT_OK;
  k_inv_sigma<<<ceil_div(k, 128), 128, 0, s>>>(evals, k, colscale, rel_floor);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_ring_core1(const float* __restrict__ u, int n1, int r0, int r1,
                             float* __restrict__ core) {
  const int total = n1 * r0 * r1;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int a = idx % r0;
    const int i = (idx / r0) % n1;
    const int b = idx / (r0 * n1);
    core[idx] = u[i + (long long)n1 * (a + r0 * b)];
  }
}

int launch_ring_core1(const float* u, int n1, int r0, int r1, float* core, cudaStream_t s) {
  const int total = n1 * r0 * r1;
  if (total <= 0) return TT_OK;
  k_ring_core1<<<ceil_div(total, 256), 256, 0, s>>>(u, n1, r0, r1, core);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

// Sign convention of every basis column: the entry of largest magnitude (lowest row on ties)
// is made positive, and column a of the FP64 companion (the small factor that produced the
// basis) is negated together with it.  TR-SVD's later unfoldings depend on these signs.
__global__ void __launch_bounds__(256) k_canon_cols(float* __restrict__ u, long long m, int r,
                                                    long long ldu, double* __restrict__ comp, int K,
                                                    long long ldc) {
  __shared__ float bv[256];
  __shared__ long long bi[256];
  __shared__ int flip;
  const int a = blockIdx.x;
  if (a >= r) return;
  float best = -1.f;
  long long besti = 0;
  for (long long i = threadIdx.x; i < m; i += blockDim.x) {
    const float v = fabsf(u[i + ldu * a]);
    if (v > best) {
      best = v;
      besti = i;
    }
  }
  bv[threadIdx.x] = best;
  bi[threadIdx.x] = besti;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const float v2 = bv[threadIdx.x + o];
      const long long i2 = bi[threadIdx.x + o];
      if (v2 > bv[threadIdx.x] || (v2 == bv[threadIdx.x] && i2 < bi[threadIdx.x])) {
        bv[threadIdx.x] = v2;
        bi[threadIdx.x] = i2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) flip = (bv[0] > 0.f && u[bi[0] + ldu * a] < 0.f) ? 1 : 0;
  __syncthreads();
  if (!flip) return;
  for (long long i = threadIdx.x; i < m; i += blockDim.x) u[i + ldu * a] = -u[i + ldu * a];
  if (comp)
    for (int k = threadIdx.x; k < K; k += blockDim.x) comp[k + ldc * a] = -comp[k + ldc * a];
}

int launch_canon_cols(float* u, long long m, int r, long long ldu, double* comp, int K,
                      long long ldc, cudaStream_t s) {
  if (r <= 0 || m <= 0) return TT_OK;
  k_canon_cols<<<r, 256, 0, s>>>(u, m, r, ldu, comp, K, ldc);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__global__ void k_check_finite(const float* __restrict__ x, long long count, int* flag) {
  int bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(x[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

int launch_check_finite(const float* x, long long count, int* flag, cudaStream_t s) {
  if (count <= 0) return TT_OK;
  k_check_finite<<<(int)std::min<long long>(ceil_div_ll(count, 256), 8LL * num_sms()), 256, 0, s>>>(
      x, count, flag);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  __syncthreads();
  return r;
}

__global__ void k_diff_norm(const float* __restrict__ x, const float* __restrict__ y,
                            long long count, double* acc) {
  __shared__ double sh[32];
  double d2 = 0.0, x2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const double xv = x[i];
    const double dv = xv - (y ? (double)y[i] : 0.0);
    d2 += dv * dv;
    x2 += xv * xv;
  }
  d2 = block_sum(d2, sh);
  x2 = block_sum(x2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&acc[0], d2);
    atomicAdd(&acc[1], x2);
  }
}

int launch_diff_norm(const float* x, const float* y, long long count, double* acc, cudaStream_t s) {
  if (count <= 0) return TT_OK;
  k_diff_norm<<<(int)std::min<long long>(ceil_div_ll(count, 256), 4LL * num_sms()), 256, 0, s>>>(
      x, y, count, acc);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

// C (M x N) = A (M x K) * B (K x N), column-major, K small.
__global__ void __launch_bounds__(256) k_gemm_nn(const float* __restrict__ a, long long M, int K,
                                                 const float* __restrict__ b, long long N,
                                                 float* __restrict__ c) {
  __shared__ float bs[32][65];
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  const long long n0 = (long long)blockIdx.y * 32;
  float acc[32];
#pragma unroll
  for (int u = 0; u < 32; ++u) acc[u] = 0.f;
  for (int k0 = 0; k0 < K; k0 += 64) {
    for (int f = threadIdx.x; f < 32 * 64; f += 256) {
      const int kk = f % 64, u = f / 64;
      const long long col = n0 + u;
      bs[u][kk] = (col < N && k0 + kk < K) ? b[(k0 + kk) + (long long)K * col] : 0.f;
    }
    __syncthreads();
    if (i < M) {
      const int kmax = (K - k0 < 64) ? K - k0 : 64;
      for (int kk = 0; kk < kmax; ++kk) {
        const float av = a[i + M * (long long)(k0 + kk)];
#pragma unroll
        for (int u = 0; u < 32; ++u) acc[u] = fmaf(av, bs[u][kk], acc[u]);
      }
    }
    __syncthreads();
  }
  if (i < M) {
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      const long long col = n0 + u;
      if (col < N) c[i + M * col] = acc[u];
    }
  }
}

int launch_gemm_nn(const float* a, long long M, int K, const float* b, long long N, float* c,
                   cudaStream_t s) {
  if (M <= 0 || N <= 0) return TT_OK;
  const long long gy = ceil_div_ll(N, 32);
  // grid.y is limited to 65535: chunk the column range.
  for (long long y0 = 0; y0 < gy; y0 += 65535) {
    const long long ny = std::min<long long>(65535, gy - y0);
    dim3 grid(ceil_div(M, 256), (unsigned)ny);
    k_gemm_nn<<<grid, 256, 0, s>>>(a, M, K, b + (long long)K * 32 * y0, N - 32 * y0,
                                   c + M * 32 * y0);
    count_launch();
    TT_LAUNCH_CHECK();
  }
  return TT_OK;
}

// err^2 += sum_{i,J} (X[i + n1 J] - sum_{a,b} G1[a + r0 i + r0 n1 b] M[b + r1 J + r1 N a])^2
__global__ void __launch_bounds__(256) k_recon_err(const float* __restrict__ x, int n1, long long N,
                                                   const float* __restrict__ g1, int r0, int r1,
                                                   const float* __restrict__ mrg, double* acc) {
  extern __shared__ float smem[];
  float* gs = smem;                     // r0*n1*r1
  const int q = r0 * r1;
  const int JT = 32;
  float* ms = gs + r0 * n1 * r1;        // JT x q: ms[jj*q + (a + r0 b)]
  __shared__ double sh[32];
  for (int f = threadIdx.x; f < r0 * n1 * r1; f += blockDim.x) gs[f] = g1[f];
  double d2 = 0.0, x2 = 0.0;
  for (long long J0 = (long long)blockIdx.x * JT; J0 < N; J0 += (long long)gridDim.x * JT) {
    __syncthreads();
    for (int f = threadIdx.x; f < JT * q; f += blockDim.x) {
      const int b = f % r1, jj = (f / r1) % JT, a = f / (r1 * JT);
      const long long J = J0 + jj;
      ms[jj * q + a + r0 * b] = (J < N) ? mrg[b + (long long)r1 * J + (long long)r1 * N * a] : 0.f;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < JT * n1; f += blockDim.x) {
      const int i = f % n1, jj = f / n1;
      const long long J = J0 + jj;
      if (J >= N) continue;
      float s = 0.f;
      for (int a = 0; a < r0; ++a)
        for (int b = 0; b < r1; ++b) s = fmaf(gs[a + r0 * i + r0 * n1 * b], ms[jj * q + a + r0 * b], s);
      const double xv = x[i + (long long)n1 * J];
      const double dv = xv - (double)s;
      d2 += dv * dv;
      x2 += xv * xv;
    }
  }
  d2 = block_sum(d2, sh);
  x2 = block_sum(x2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&acc[0], d2);
    atomicAdd(&acc[1], x2);
  }
}

int launch_recon_err(const float* x, int n1, long long N, const float* g1, int r0, int r1,
                     const float* mrg, double* acc, cudaStream_t s) {
  const size_t shm = ((size_t)r0 * n1 * r1 + 32 * (size_t)r0 * r1) * sizeof(float);
  if (shm > 200 * 1024) {
    set_error(TT_ERR_UNSUPPORTED, "reconstruction check: first core too large");
    return TT_ERR_UNSUPPORTED;
  }
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_recon_err, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const int grid = (int)std::min<long long>(ceil_div_ll(N, 32), 8LL * num_sms());
  k_recon_err<<<grid, 256, shm, s>>>(x, n1, N, g1, r0, r1, mrg, acc);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

}  // namespace ttr
