// CUDA-core kernels: the plain-FP32 GEMM engine and every small linear-algebra kernel of the
// TT/TR-SVD chain (Gaussian test matrix, Gram matrices, CholeskyQR2, Jacobi eigen-solver,
// bond permute, core folding, reconstruction error).
#include <float.h>
#include <stdlib.h>
#include <math.h>

#include <algorithm>

#include "kernels.cuh"
#include "philox.cuh"
#include "jacobi_rot.cuh"
#include "bl_solver.cuh"

namespace ttr {

thread_local int g_kernel_launches = 0;

static int num_sms() { return dev_sms(); }
static int max_optin_smem();

// ---------------------------------------------------------------------------------------
// Philox4x32-10 Gaussian generator (replaces curandGenerateNormal, TT3O:585-587)
// ---------------------------------------------------------------------------------------

__global__ void k_gaussian(float* __restrict__ out, long long rows, long long total, long long ld,
                           unsigned long long seed, unsigned stream_id) {
  const long long ncall = (total + 3) / 4;
  if (ld == rows) {
    // contiguous matrix: element e sits at out[e]; whole float4 stores when aligned
    const bool v4 = (total & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncall;
         c += (long long)gridDim.x * blockDim.x) {
      const float4 gv = philox_normal4((unsigned long long)c, stream_id, seed);
      if (v4) {
        reinterpret_cast<float4*>(out)[c] = gv;
      } else {
        const float g[4] = {gv.x, gv.y, gv.z, gv.w};
#pragma unroll
        for (int l = 0; l < 4; ++l)
          if (4 * c + l < total) out[4 * c + l] = g[l];
      }
    }
    return;
  }
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncall;
       c += (long long)gridDim.x * blockDim.x) {
    const float4 gv = philox_normal4((unsigned long long)c, stream_id, seed);
    const float g[4] = {gv.x, gv.y, gv.z, gv.w};
    // element e = row + rows * col; one 64-bit division per call, then step through rows
    long long col = (4 * c) / rows;
    long long row = 4 * c - col * rows;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      if (4 * c + l < total) out[row + ld * col] = g[l];
      if (++row == rows) {
        row = 0;
        ++col;
      }
    }
  }
}

// Rows [row0, row0 + nrows) of the (total_rows x cols) matrix k_gaussian generates (its element
// (i, c) is component e % 4 of Philox call e / 4, e = i + total_rows * c): the block of a
// column-sharded Omega that one rank multiplies with its columns.
__global__ void k_gaussian_rows(float* __restrict__ out, long long row0, long long nrows, long long total_rows,
                                int cols, long long ld, unsigned long long seed, unsigned stream_id) {
  const long long total = nrows * cols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long c = idx / nrows, i = idx - c * nrows;
    const long long e = row0 + i + total_rows * c;
    const float4 g = philox_normal4((unsigned long long)(e >> 2), stream_id, seed);
    const int l = (int)(e & 3);
    out[i + ld * c] = l == 0 ? g.x : l == 1 ? g.y : l == 2 ? g.z : g.w;
  }
}

int launch_gaussian_rows(float* out, long long row0, long long nrows, long long total_rows, int cols, long long ld,
                         unsigned long long seed, unsigned stream_id, cudaStream_t s) {
  const long long total = nrows * (long long)cols;
  if (total <= 0) return TT_OK;
  k_gaussian_rows<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0, s>>>(
      out, row0, nrows, total_rows, cols, ld, seed, stream_id);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
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
// Asynchronous global -> shared copies (cp.async): 16-byte, and 4-byte with zero fill when
// `valid` is false (no byte is read then).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// 32 x RI rows of A per block (RI per thread) x NT sketch columns (NT / 8 per thread); narrow
// sketches (NT <= 24) take RI = 16 rows per thread, so that each shared-memory load feeds more
// FMAs.  The long dimension runs in chunks of JC columns of A (32 KB of A per chunk) streamed
// through a 3-stage shared-memory ring by cp.async (two chunks in flight while the third is
// multiplied: the loads need no registers), one barrier per chunk.  Products by paired FP32 FMAs
// (fma.rn.f32x2, each lane rounded like fmaf), the row pairs straight from 16-byte shared loads;
// W's rows are padded to NT + 1 words so its copies (JC consecutive rows per warp) hit distinct
// banks.  Split partials are written in FP64.
constexpr int kSkStages = 3;
template <int NT>
struct SkTile {
  static constexpr int RI = NT <= 24 ? 16 : 8;  // rows per thread
  static constexpr int TI = 32 * RI;             // rows per block
  static constexpr int JC = 8192 / TI;           // columns of A per chunk (TI x JC = 8192 floats)
  static constexpr int NTP = NT + 1;             // padded row of W in shared memory
  static constexpr size_t smem = (size_t)kSkStages * (TI * JC + JC * NTP) * sizeof(float);
};
template <int NT>
constexpr size_t sk_smem() { return SkTile<NT>::smem; }

template <int NT>
__global__ void __launch_bounds__(256, NT >= 40 ? 1 : 2) k_sketch_simt(const float* __restrict__ a, long long m,
                                                                       long long n, const float* __restrict__ w,
                                                                       int N, long long wj, long long wc,
                                                                       long long jchunk, int cblk,
                                                                       double* __restrict__ part) {
  using T = SkTile<NT>;
  constexpr int RI = T::RI, TI = T::TI, JC = T::JC, NTP = T::NTP, RC = NT / 8;
  constexpr int AV = (TI * JC / 4) / 256;     // 16-byte copies of A per thread per chunk
  constexpr int WV = (JC * NT + 255) / 256;   // W values per thread per chunk
  extern __shared__ __align__(16) float sm_sk[];
  float* as_base = sm_sk;                            // [ST][JC][TI]
  float* ws_base = sm_sk + kSkStages * JC * TI;      // [ST][JC][NTP]
  const int tid = threadIdx.x;
  const long long i0 = (long long)blockIdx.x * TI;
  const int split = blockIdx.y;
  const int c0 = blockIdx.z * NT;
  const long long jb = (long long)split * jchunk;
  const long long je = (jb + jchunk < n) ? jb + jchunk : n;
  const int ti = tid >> 3, tc = tid & 7;
  // accumulators paired over rows: acc2[p][c] = (acc[2p][c], acc[2p + 1][c])
  uint64_t acc2[RI / 2][RC];
#pragma unroll
  for (int e = 0; e < RI / 2; ++e)
#pragma unroll
    for (int c = 0; c < RC; ++c) acc2[e][c] = 0ull;
  const bool vec = ((m & 3) == 0) && ((((uintptr_t)a) & 15) == 0);
  const int nchunks = je > jb ? (int)((je - jb + JC - 1) / JC) : 0;
  // Copies of chunk t into ring slot t % ST (one commit group per chunk, empty past the end).
  auto fill = [&](int t) {
    if (t < nchunks) {
      const long long j0 = jb + (long long)t * JC;
      float* as = as_base + (t % kSkStages) * JC * TI;
      float* wsm = ws_base + (t % kSkStages) * JC * NTP;
#pragma unroll
      for (int q = 0; q < AV; ++q) {
        const int f = tid + 256 * q;
        const int jj = f / (TI / 4), i4 = f % (TI / 4);
        const long long j = j0 + jj, i = i0 + 4 * i4;
        float* dst = &as[jj * TI + 4 * i4];
        const float* src = a + j * m + i;
        if (j < je && vec && i + 3 < m) {
          cp_async16(dst, src);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const bool ok = j < je && i + e < m;
            cp_async4(dst + e, ok ? src + e : a, ok);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < WV; ++u) {
        const int f = tid + 256 * u;
        if (f < JC * NT) {
          int jj, c;
          if (wc == 1) {
            c = f % NT;
            jj = f / NT;
          } else {
            jj = f % JC;
            c = f / JC;
          }
          const long long j = j0 + jj;
          const bool ok = j < je && c0 + c < N;
          cp_async4(&wsm[jj * NTP + c], ok ? w + j * wj + (long long)(c0 + c) * wc : w, ok);
        }
      }
    }
    cp_async_commit();
  };
  fill(0);
  fill(1);
  for (int t = 0; t < nchunks; ++t) {
    cp_async_wait<kSkStages - 2>();  // this thread's copies of chunk t have landed
    __syncthreads();                 // everyone's have; slot (t + 2) % ST was last read at t - 1
    fill(t + 2);
    const float* as = as_base + (t % kSkStages) * JC * TI;
    const float* wsm = ws_base + (t % kSkStages) * JC * NTP;
#pragma unroll
    for (int jj = 0; jj < JC; ++jj) {
      uint64_t xp[RI / 2];
#pragma unroll
      for (int q = 0; q < RI / 4; ++q) {
        const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(&as[jj * TI + ti * RI + 4 * q]);
        xp[2 * q] = x.x;
        xp[2 * q + 1] = x.y;
      }
#pragma unroll
      for (int c = 0; c < RC; ++c) {
        const uint64_t wd = f2_dup(wsm[jj * NTP + tc * RC + c]);
#pragma unroll
        for (int e = 0; e < RI / 2; ++e) ffma2(acc2[e][c], xp[e], wd);
      }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int e = 0; e < RI; ++e) {
    const long long i = i0 + ti * RI + e;
#pragma unroll
    for (int c = 0; c < RC; ++c) {
      const int col = c0 + tc * RC + c;
      float lo, hi;
      f2_unpack(acc2[e >> 1][c], lo, hi);
      if (i < m && col < N) part[((long long)split * N + col) * m + i] = (double)((e & 1) ? hi : lo);
    }
  }
  (void)cblk;
}

// Launch of k_sketch_simt with the tile width covering N (multiples of 8 up to 64; wider N
// takes several column blocks of 64).
static void launch_sketch_simt_kernel(const float* a, long long m, long long n, const float* w, int N, long long wj,
                                      long long wc, long long jchunk, int nsplit, double* part, cudaStream_t s) {
  const int NT = N <= 16 ? 16 : N <= 24 ? 24 : N <= 32 ? 32 : N <= 40 ? 40 : N <= 48 ? 48 : 64;
  const int cblk = ceil_div(N, NT);
  const int TI = NT <= 24 ? SkTile<16>::TI : SkTile<64>::TI;
  dim3 grid(ceil_div(m, TI), nsplit, cblk);
  const size_t shm = NT == 16 ? sk_smem<16>() : NT == 24 ? sk_smem<24>() : NT == 32 ? sk_smem<32>()
                   : NT == 40 ? sk_smem<40>() : NT == 48 ? sk_smem<48>() : sk_smem<64>();
#define SK_ATTR(V) smem_optin_k(k_sketch_simt<V>, sk_smem<V>())
  SK_ATTR(16); SK_ATTR(24); SK_ATTR(32); SK_ATTR(40); SK_ATTR(48); SK_ATTR(64);
#undef SK_ATTR
#define SK_CASE(V) \
  case V: k_sketch_simt<V><<<grid, 256, shm, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
  switch (NT) {
    SK_CASE(16)
    SK_CASE(24)
    SK_CASE(32)
    SK_CASE(40)
    SK_CASE(48)
    default: k_sketch_simt<64><<<grid, 256, shm, s>>>(a, m, n, w, N, wj, wc, jchunk, cblk, part); break;
  }
#undef SK_CASE
}

// Sum of nsplit partial blocks: each 256-thread block owns 32 consecutive outputs, its 8 warps
// read interleaved splits (coalesced 256-byte rows, several loads in flight per lane) and the
// 8 warp sums are added in a fixed order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(256) k_reduce_splits(const double* __restrict__ part, long long count,
                                                       int nsplit, double* __restrict__ y) {
  __shared__ double red[8][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long base = (long long)blockIdx.x * 32; base < count; base += (long long)gridDim.x * 32) {
    const long long idx = base + lane;
    double s0 = 0.0, s1 = 0.0;
    if (idx < count) {
      int k = warp;
      for (; k + 8 < nsplit; k += 16) {
        s0 += part[(long long)k * count + idx];
        s1 += part[(long long)(k + 8) * count + idx];
      }
      if (k < nsplit) s0 += part[(long long)k * count + idx];
    }
    red[warp][lane] = s0 + s1;
    __syncthreads();
    if (warp == 0 && idx < count) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) t += red[w][lane];
      y[idx] = t;
    }
    __syncthreads();
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
  k_reduce_splits<<<(int)std::min<long long>(ceil_div_ll(count, 32), 16LL * num_sms()), 256, 0, s>>>(
      part, count, nsplit, y);
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
  launch_sketch_simt_kernel(a, m, n, w, N, wj, wc, jchunk, nsplit, part, s);
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
  launch_sketch_simt_kernel(a, m, n, w, N, wj, wc, jchunk, nsplit, part, s);
  count_launch();
  TT_LAUNCH_CHECK();
  return launch_reduce_splits(part, (long long)N * m, nsplit, y, s);
}

// ---------------------------------------------------------------------------------------
// Plain-FP32 projection  out = A^T Q  (A column-major m x n, contraction over m)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int swz(int row, int col) { return col ^ (((row >> 2) & 7) << 2); }

// 256 columns of A per block (8 per thread) x NT outputs (NT / 8 per thread), K in chunks of
// 32: the next chunk is loaded into registers while the current one is multiplied out of
// shared memory (two buffers, one barrier per chunk).
template <int NT>
__global__ void __launch_bounds__(256, NT >= 64 ? 1 : 2) k_project_simt(const float* __restrict__ a, long long m,
                                                                        long long n, const float* __restrict__ q,
                                                                        int N, long long ldq, float* __restrict__ out,
                                                                        long long ldo, int mode, int r0, int r1,
                                                                        long long kchunk) {
  constexpr int TJ = 256, KC = 32, RJ = 8, RC = NT / 8;
  constexpr int AV = (TJ * KC / 4) / 256;    // float4 loads of A per thread per chunk
  constexpr int QV = (KC * NT + 255) / 256;  // Q values per thread per chunk
  extern __shared__ __align__(16) float sm_ps[];
  float* as_base = sm_ps;                // [2][KC][TJ]
  float* qs_base = sm_ps + 2 * KC * TJ;  // [2][KC][NT]
  const int tid = threadIdx.x;
  const long long j0 = (long long)blockIdx.x * TJ;
  const int c0 = blockIdx.y * NT;
  const int tj = tid >> 3, tc = tid & 7;
  // accumulators paired over output rows (fma.rn.f32x2), as in k_sketch_simt
  uint64_t acc2[RJ / 2][RC];
#pragma unroll
  for (int e = 0; e < RJ / 2; ++e)
#pragma unroll
    for (int c = 0; c < RC; ++c) acc2[e][c] = 0ull;
  const bool vec = ((m & 3) == 0) && ((((uintptr_t)a) & 15) == 0);
  // K range of this split (blockIdx.z); the split's output block is out + z * n * ldo.
  const long long kb = (long long)blockIdx.z * kchunk;
  const long long ke = (kb + kchunk < m) ? kb + kchunk : m;
  out += (long long)blockIdx.z * n * ldo;
  float4 ra[AV];
  float rq[QV];
  auto fetch = [&](long long k0) {
#pragma unroll
    for (int qq = 0; qq < AV; ++qq) {
      const int f = tid + 256 * qq;
      const int jj = f >> 3, k4 = f & 7;
      const long long j = j0 + jj, k = k0 + 4 * k4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j < n) {
        const float* p = a + j * m + k;
        if (vec && k + 3 < ke) {
          v = __ldg(reinterpret_cast<const float4*>(p));
        } else {
          if (k < ke) v.x = p[0];
          if (k + 1 < ke) v.y = p[1];
          if (k + 2 < ke) v.z = p[2];
          if (k + 3 < ke) v.w = p[3];
        }
      }
      ra[qq] = v;
    }
#pragma unroll
    for (int u = 0; u < QV; ++u) {
      const int f = tid + 256 * u;
      const int kk = f % KC, c = f / KC;
      const long long k = k0 + kk;
      rq[u] = (f < KC * NT && k < ke && c0 + c < N) ? q[k + ldq * (long long)(c0 + c)] : 0.f;
    }
  };
  auto stash = [&](int b) {
    float* as = as_base + b * KC * TJ;
    float* qs = qs_base + b * KC * NT;
#pragma unroll
    for (int qq = 0; qq < AV; ++qq) {
      const int f = tid + 256 * qq;
      const int jj = f >> 3, kk = 4 * (f & 7);
      as[(kk + 0) * TJ + swz(kk + 0, jj)] = ra[qq].x;
      as[(kk + 1) * TJ + swz(kk + 1, jj)] = ra[qq].y;
      as[(kk + 2) * TJ + swz(kk + 2, jj)] = ra[qq].z;
      as[(kk + 3) * TJ + swz(kk + 3, jj)] = ra[qq].w;
    }
#pragma unroll
    for (int u = 0; u < QV; ++u) {
      const int f = tid + 256 * u;
      if (f < KC * NT) qs[(f % KC) * NT + f / KC] = rq[u];
    }
  };
  if (kb < ke) {
    fetch(kb);
    stash(0);
  }
  __syncthreads();
  int b = 0;
  for (long long k0 = kb; k0 < ke; k0 += KC) {
    const bool more = k0 + KC < ke;
    if (more) fetch(k0 + KC);
    const float* as = as_base + b * KC * TJ;
    const float* qs = qs_base + b * KC * NT;
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      const ulonglong2 x0 = *reinterpret_cast<const ulonglong2*>(&as[kk * TJ + swz(kk, tj * RJ)]);
      const ulonglong2 x1 = *reinterpret_cast<const ulonglong2*>(&as[kk * TJ + swz(kk, tj * RJ + 4)]);
      const uint64_t xp[4] = {x0.x, x0.y, x1.x, x1.y};
#pragma unroll
      for (int c = 0; c < RC; ++c) {
        const uint64_t qd = f2_dup(qs[kk * NT + tc * RC + c]);
#pragma unroll
        for (int e = 0; e < RJ / 2; ++e) ffma2(acc2[e][c], xp[e], qd);
      }
    }
    if (more) stash(b ^ 1);
    __syncthreads();
    b ^= 1;
  }
#pragma unroll
  for (int e = 0; e < RJ; ++e) {
    const long long j = j0 + tj * RJ + e;
    if (j >= n) continue;
#pragma unroll
    for (int c = 0; c < RC; ++c) {
      const int col = c0 + tc * RC + c;
      if (col >= N) continue;
      float lo, hi;
      f2_unpack(acc2[e >> 1][c], lo, hi);
      const float v = (e & 1) ? hi : lo;
      if (mode == OUT_ROWMAJOR) {
        out[j * ldo + col] = v;
      } else if (mode == OUT_COLMAJOR) {
        out[j + ldo * col] = v;
      } else {
        const int ai = col % r0, bi = col / r0;
        out[(long long)bi + (long long)r1 * (j + n * (long long)ai)] = v;
      }
    }
  }
}

// Small-K projection out = Q^T A for K = m <= 64 (the rotation E_r^T B of a small factor, or
// an m <= 64 unfolding).  A's columns are contiguous, so a tile of TJ columns is one contiguous
// block: it is staged through shared memory with coalesced float4 loads (odd row stride,
// conflict-free), Q sits in shared memory as float4 rows, and each column's NP outputs are
// computed by SPLIT threads (NP / SPLIT each, which keeps registers low enough for several
// blocks per SM).  Row-major outputs and the TR bond permute leave through shared memory as
// contiguous runs.
template <int NP, int SPLIT>
__global__ void __launch_bounds__(256) k_proj_smallk(const float* __restrict__ a, int m, long long n,
                                                     const float* __restrict__ q, int N, long long ldq,
                                                     float* __restrict__ out, long long ldo, int mode,
                                                     int r0, int r1) {
  constexpr int TJ = 256 / SPLIT;   // columns per tile
  constexpr int NPT = NP / SPLIT;   // outputs per thread
  static_assert(NPT % 4 == 0, "outputs per thread");
  extern __shared__ __align__(16) float sm_pk[];
  float* Es = sm_pk;            // m x NP: Es[k * NP + c] = Q[k + ldq c]
  float* Xs = Es + 64 * NP;     // TJ x S input tile, then TJ x (NP + 1) output tile
  const int S = (m & 1) ? m : m + 1;
  constexpr int OS = NP + 1;
  const int tid = threadIdx.x;
  const int col_t = tid % TJ, grp = tid / TJ;
  for (int idx = tid; idx < m * NP; idx += 256) {
    const int k = idx / NP, c = idx - (idx / NP) * NP;
    Es[idx] = (c < N) ? q[k + ldq * (long long)c] : 0.f;
  }
  const bool vec = (m & 3) == 0 && ((reinterpret_cast<uintptr_t>(a) & 15) == 0);
  // Row-major outputs with ldo == N form one contiguous block per tile; bond-permuted outputs
  // (r0, r1, n) -> (r1, n, r0) form r0 contiguous runs of r1 * nj values per tile.
  const bool staged_out = (mode == OUT_ROWMAJOR && ldo == N) || (mode == OUT_PERM231 && r0 * r1 == N);
  // Quotients of tile-local indices (< 2^15) by m, N or r1 (<= 128) through a float reciprocal:
  // the rounding error is far below the 0.5 / divisor margin, so the floor is exact.
  const float inv_m = 1.0f / (float)m, inv_n = 1.0f / (float)N, inv_r1 = 1.0f / (float)(r1 > 0 ? r1 : 1);
  auto qdiv = [](int e, float inv) { return (int)(((float)e + 0.5f) * inv); };
  for (long long tile = blockIdx.x; tile * TJ < n; tile += gridDim.x) {
    const long long j0 = tile * TJ;
    const int nj = (int)((n - j0 < TJ) ? n - j0 : TJ);
    const float* src = a + j0 * m;
    const int cnt = nj * m;
    __syncthreads();
    if (vec) {
      for (int f4 = tid; f4 < (cnt >> 2); f4 += 256) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(src) + f4);
        const int e = 4 * f4, col = qdiv(e, inv_m), k = e - col * m;
        float* d = Xs + col * S + k;
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
      }
    } else {
      for (int f = tid; f < cnt; f += 256) {
        const int col = qdiv(f, inv_m), k = f - col * m;
        Xs[col * S + k] = __ldg(src + f);
      }
    }
    __syncthreads();
    float acc[NPT];
#pragma unroll
    for (int c = 0; c < NPT; ++c) acc[c] = 0.f;
    if (col_t < nj) {
      const float* xr = Xs + col_t * S;
      for (int k = 0; k < m; ++k) {
        const float x = xr[k];
        const float4* er = reinterpret_cast<const float4*>(Es + k * NP + grp * NPT);
#pragma unroll
        for (int c4 = 0; c4 < NPT / 4; ++c4) {
          const float4 e = er[c4];
          acc[4 * c4] = fmaf(x, e.x, acc[4 * c4]);
          acc[4 * c4 + 1] = fmaf(x, e.y, acc[4 * c4 + 1]);
          acc[4 * c4 + 2] = fmaf(x, e.z, acc[4 * c4 + 2]);
          acc[4 * c4 + 3] = fmaf(x, e.w, acc[4 * c4 + 3]);
        }
      }
    }
    if (staged_out) {
      __syncthreads();
      if (col_t < nj) {
#pragma unroll
        for (int c = 0; c < NPT; ++c)
          if (grp * NPT + c < N) Xs[col_t * OS + grp * NPT + c] = acc[c];
      }
      __syncthreads();
      if (mode == OUT_ROWMAJOR) {
        float* dst = out + j0 * N;
        for (int f = tid; f < nj * N; f += 256) {
          const int col = qdiv(f, inv_n), c = f - col * N;
          dst[f] = Xs[col * OS + c];
        }
      } else {
        const int run = r1 * nj;
        for (int ai = 0; ai < r0; ++ai) {
          float* dst = out + (long long)r1 * (j0 + n * (long long)ai);
          for (int f = tid; f < run; f += 256) {
            const int col = qdiv(f, inv_r1), bi = f - col * r1;
            dst[f] = Xs[col * OS + ai + r0 * bi];
          }
        }
      }
    } else if (col_t < nj) {
      const long long j = j0 + col_t;
#pragma unroll
      for (int cc = 0; cc < NPT; ++cc) {
        const int c = grp * NPT + cc;
        if (c >= N) continue;
        if (mode == OUT_ROWMAJOR) {
          out[j * ldo + c] = acc[cc];
        } else if (mode == OUT_COLMAJOR) {
          out[j + ldo * c] = acc[cc];
        } else {
          const int ai = c % r0, bi = c / r0;
          out[(long long)bi + (long long)r1 * (j + n * (long long)ai)] = acc[cc];
        }
      }
    }
  }
}

// Sum of the K-split partial projections (row-major n x N blocks) into the requested layout.
__global__ void k_project_reduce(const float* __restrict__ part, long long n, int N, int nsplit,
                                 float* __restrict__ out, long long ldo, int mode, int r0, int r1) {
  const long long total = n * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    float v = 0.f;
    for (int z = 0; z < nsplit; ++z) v += part[(long long)z * total + idx];
    const long long j = idx / N;
    const int c = (int)(idx - j * N);
    if (mode == OUT_ROWMAJOR) {
      out[j * ldo + c] = v;
    } else if (mode == OUT_COLMAJOR) {
      out[j + ldo * c] = v;
    } else {
      const int ai = c % r0, bi = c / r0;
      out[(long long)bi + (long long)r1 * (j + n * (long long)ai)] = v;
    }
  }
}

namespace {
constexpr size_t kProjectSplitCap = 16u << 20;  // bytes of K-split partials

// K splits for projections whose column tiles alone cannot fill the GPU.
int project_ksplit(long long m, long long n, int N, long long* kchunk) {
  const int NT = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  const long long blocks = ceil_div_ll(n, 256) * ceil_div_ll(N, NT);
  int ks = 1;
  if (m >= 256 && blocks < 2LL * num_sms()) {
    ks = (int)std::min<long long>(ceil_div_ll(2LL * num_sms(), blocks), m / 64);
    const long long cap = (long long)(kProjectSplitCap / (sizeof(float) * (size_t)n * N));
    ks = (int)std::max<long long>(1, std::min<long long>(ks, cap));
  }
  long long kc = ceil_div_ll(m, ks);
  kc = ceil_div_ll(kc, 32) * 32;
  *kchunk = kc;
  return (int)ceil_div_ll(m, kc);
}
}  // namespace

size_t project_ws_bytes(long long m, long long n, int N) {
  long long kc;
  const int ks = project_ksplit(m, n, N, &kc);
  const size_t split = ks > 1 ? (size_t)ks * n * N * sizeof(float) : 0;
  return split + 2 * (size_t)m * N * sizeof(float) + 4096;
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
  if (m <= 64 && N <= 64) {
    // SPLIT threads per column: 1 for NP = 16, 2 for 32 and 48, 4 for 64.
    const int split = NT <= 16 ? 1 : NT <= 48 ? 2 : 4;
    const int tj = 256 / split;
    const size_t shm = (64 * (size_t)NT + (size_t)tj * std::max<long long>(m + 1, NT + 1)) * sizeof(float);
    smem_optin_k(k_proj_smallk<16, 1>, 100 * 1024);
    smem_optin_k(k_proj_smallk<32, 2>, 100 * 1024);
    smem_optin_k(k_proj_smallk<48, 2>, 100 * 1024);
    smem_optin_k(k_proj_smallk<64, 4>, 100 * 1024);
    const int grid = (int)std::min<long long>(ceil_div_ll(n, tj), 64LL * num_sms());
    const int mi = (int)m;
    switch (NT) {
      case 16: k_proj_smallk<16, 1><<<grid, 256, shm, s>>>(a, mi, n, q, N, ldq, out, ldo, mode, r0, r1); break;
      case 32: k_proj_smallk<32, 2><<<grid, 256, shm, s>>>(a, mi, n, q, N, ldq, out, ldo, mode, r0, r1); break;
      case 48: k_proj_smallk<48, 2><<<grid, 256, shm, s>>>(a, mi, n, q, N, ldq, out, ldo, mode, r0, r1); break;
      default: k_proj_smallk<64, 4><<<grid, 256, shm, s>>>(a, mi, n, q, N, ldq, out, ldo, mode, r0, r1); break;
    }
    count_launch();
    TT_LAUNCH_CHECK();
    return TT_OK;
  }
  long long kc;
  int ks = project_ksplit(m, n, N, &kc);
  float* part = nullptr;
  const size_t mk = ws.mark();
  if (ks > 1) {
    part = ws.take<float>((size_t)ks * n * N);
    if (!part) {
      ks = 1;
      kc = m;
    }
  } else {
    kc = m;
  }
  // output tile width: the smallest multiple of 8 in {16, 24, 32, 40, 48, 64} covering N
  const int NTs = N <= 16 ? 16 : N <= 24 ? 24 : N <= 32 ? 32 : N <= 40 ? 40 : N <= 48 ? 48 : 64;
  dim3 grid(ceil_div(n, 256), ceil_div(N, NTs), ks);
  float* dst = ks > 1 ? part : out;
  const long long ldd = ks > 1 ? N : ldo;
  const int md = ks > 1 ? OUT_ROWMAJOR : mode;
#define PS_ATTR(V) smem_optin_k(k_project_simt<V>, (size_t)2 * 32 * (256 + V) * 4)
  PS_ATTR(16); PS_ATTR(24); PS_ATTR(32); PS_ATTR(40); PS_ATTR(48); PS_ATTR(64);
#undef PS_ATTR
  const size_t pshm = (size_t)2 * 32 * (256 + NTs) * sizeof(float);
#define PS_CASE(V) \
  case V: k_project_simt<V><<<grid, 256, pshm, s>>>(a, m, n, q, N, ldq, dst, ldd, md, r0, r1, kc); break;
  switch (NTs) {
    PS_CASE(16)
    PS_CASE(24)
    PS_CASE(32)
    PS_CASE(40)
    PS_CASE(48)
    default: k_project_simt<64><<<grid, 256, pshm, s>>>(a, m, n, q, N, ldq, dst, ldd, md, r0, r1, kc); break;
  }
#undef PS_CASE
  count_launch();
  TT_LAUNCH_CHECK();
  if (ks > 1) {
    const long long total = n * N;
    k_project_reduce<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0, s>>>(
        part, n, N, ks, out, ldo, mode, r0, r1);
    count_launch();
    TT_LAUNCH_CHECK();
  }
  ws.reset(mk);
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

// W = sum over the per-block partials (upper tiles of size T stored, the lower half mirrored):
// one warp per entry, lanes stride over the blocks, fixed-order shuffle tree (deterministic).
__global__ void k_gram_reduce(const double* __restrict__ part, int nblk, int MP, int M, int T,
                              double* __restrict__ w) {
  const int idx = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (idx >= M * M) return;
  const int aI = idx % M, bI = idx / M;
  const int src = (aI / T <= bI / T) ? aI * MP + bI : bI * MP + aI;
  double sacc = 0.0;
  for (int k = lane; k < nblk; k += 32) sacc += part[(long long)k * MP * MP + src];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
  if (lane == 0) w[aI + (long long)M * bI] = sacc;
}

static void launch_gram_reduce(const double* part, int nblk, int MP, int M, int T, double* w, cudaStream_t s) {
  const long long threads = 32LL * M * M;
  k_gram_reduce<<<(int)ceil_div_ll(threads, 256), 256, 0, s>>>(part, nblk, MP, M, T, w);
}

// ---------------------------------------------------------------------------------------
// Gram of many short vectors  W = sum_j x_j x_j^T  (17 <= M <= 64 components), two layouts:
//  * contiguous (COL = false): x_j = x + j M, M % 4 == 0, x 16-byte aligned -- the Gram of a
//    long unfolding with few rows (columns contiguous) and of a row-major factor B^T.  A stage
//    of VC vectors is one contiguous block, copied with 16-byte cp.async;
//  * column-major (COL = true): component c of x_j at x[j + c ld] -- a tall n x M matrix (the
//    power-iteration basis Z).  Each component's VC values are copied with 16-byte cp.async
//    into a row of the stage, chunks swizzled for conflict-free column reads (gv_col_at).
// Stages are NS deep.  Each warp computes a 32 x 32 block of W: lane (p, q) = (lane / 8,
// lane % 8) holds rows 8p..8p+7 x columns 4q..4q+3, 12 loaded values per vector for 32 FMAs.
// MP = 32 has one such block (12 warps split the vectors), MP = 64 the three upper blocks
// (4 warps each); one block of 384 threads per SM.  Rows and columns >= M read neighbouring
// words; those entries are never written out.  FP32 products accumulate over VFLUSH vectors
// per lane (round-to-nearest FMA, unbiased) and are then added into FP64; ACC64 accumulates
// every product in FP64 instead.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem) : "memory");
}

constexpr int GV_VC = 192;  // vectors per stage
constexpr int GV_NS = 4;    // stages in flight
constexpr int GV_VFLUSH = 64;

// Column-major stages: component c's values of the stage's vectors occupy row c (stride
// GV_VC floats) with 4-vector chunks XOR-swizzled by the key (c >> 2) & 7, so the 16-byte copies
// stay aligned and the reads of the rows 8p + i (i fixed) and 4q + j (j fixed) of one vector hit
// distinct banks.  Element (c, v) of the stage sits at gv_col_at(c, v).
__device__ __forceinline__ int gv_col_key(int c) { return ((c >> 2) & 7) << 2; }
__device__ __forceinline__ int gv_col_at(int c, int v) { return c * GV_VC + (v ^ gv_col_key(c)); }

// Copy vectors [v0, v0 + nv) of the column-major n x M matrix x (column stride ld) into a
// column-major stage: 16-byte copies of 4 vectors when the layout allows them, 4-byte ones
// otherwise.
template <int NT>
__device__ __forceinline__ void gv_load_col(float* dst, const float* __restrict__ x, long long v0, int nv, int M,
                                            long long ld, int tid) {
  const bool v16 = ((ld & 3) == 0) && ((v0 & 3) == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  const int n4 = v16 ? nv >> 2 : 0;  // whole 4-vector chunks per component
  if (n4 > 0) {
    const int tot = n4 * M;
    const float inv = 1.0f / (float)n4;  // exact quotients: c < 64, far inside the 0.5 / n4 margin
    for (int f = tid; f < tot; f += NT) {
      const int c = (int)(((float)f + 0.5f) * inv), g = f - c * n4;
      cp_async16(dst + gv_col_at(c, 4 * g), x + (v0 + 4 * g) + (long long)c * ld);
    }
  }
  const int rest = nv - 4 * n4;  // remaining vectors, 4-byte copies
  if (rest > 0) {
    const int tot = rest * M;
    const float inv = 1.0f / (float)rest;
    for (int f = tid; f < tot; f += NT) {
      const int c = (int)(((float)f + 0.5f) * inv), v = 4 * n4 + (f - c * rest);
      cp_async4(dst + gv_col_at(c, v), x + (v0 + v) + (long long)c * ld);
    }
  }
}

template <int MP>
struct GramVecShape {
  static constexpr int WB = MP == 32 ? 1 : 3;    // 32 x 32 warp blocks (upper triangle)
  static constexpr int WPB = MP == 32 ? 12 : 4;  // warps per warp block
  static constexpr int NT = 32 * WB * WPB;       // 384
};

// FP64 products of row-major vectors convert each stage to FP64 once, in shared memory, next to
// two FP32 stages (the conversion is the scarce unit: F2F runs at a fraction of the FP64 FMA
// rate, and converting per use costs every lane 12 conversions per 32 products).
static size_t gram_vec_smem(int MP, int M, bool col, bool acc64 = false) {
  const size_t stage = col ? (size_t)MP * GV_VC : (size_t)GV_VC * M + MP;
  const size_t red = (size_t)12 * 1024 * 2;  // per-warp 32 x 32 FP64 blocks, in floats
  if (acc64 && !col) return std::max(stage * 2 + ((size_t)GV_VC * M + MP) * 2, red) * sizeof(float);
  return std::max(stage * GV_NS, red) * sizeof(float);
}

template <int MP, bool ACC64, bool COL>
__global__ void __launch_bounds__(GramVecShape<MP>::NT, 1) k_gram_vec(const float* __restrict__ x, long long nvec,
                                                                    int M, long long ld, long long vchunk,
                                                                    double* __restrict__ part) {
  using S = GramVecShape<MP>;
  constexpr bool CONV = ACC64 && !COL;    // stages converted to FP64 once
  constexpr int NS = CONV ? 2 : GV_NS;    // FP32 stages
  extern __shared__ __align__(16) float sm_gv[];
  // floats per stage buffer: COL, MP component rows; otherwise VC vectors + MP words of slack
  const int stage_f = COL ? MP * GV_VC : GV_VC * M + MP;
  // CONV: VC x M doubles + MP of slack (rows >= M of the last vector read past its end)
  double* dbuf = reinterpret_cast<double*>(sm_gv + NS * stage_f);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wb = warp % S::WB, ph = warp / S::WB;
  const int r0 = (wb == 2 ? 32 : 0) + 8 * (lane >> 3);
  const int c0 = (wb == 0 ? 0 : 32) + 4 * (lane & 7);
  const long long vb = (long long)blockIdx.x * vchunk;
  const long long ve = (vb + vchunk < nvec) ? vb + vchunk : nvec;
  const long long nst = vb < ve ? (ve - vb + GV_VC - 1) / GV_VC : 0;

  auto load = [&](long long st) {
    const long long v0 = vb + st * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    float* dst = sm_gv + (int)(st % NS) * stage_f;
    if (COL) {
      gv_load_col<S::NT>(dst, x, v0, nv, M, ld, tid);
    } else {
      const int n16 = nv * M / 4;
      const float* src = x + v0 * M;
      for (int f = tid; f < n16; f += S::NT) cp_async16(dst + 4 * f, src + 4 * f);
    }
  };

  float acc[8][4];
  double accd[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[i][j] = 0.f;
      accd[i][j] = 0.0;
    }
  int since = 0;
#pragma unroll
  for (int st = 0; st < NS - 1; ++st) {
    if (st < nst) load(st);
    cp_async_commit();
  }
  for (long long it = 0; it < nst; ++it) {
    cp_async_wait<NS - 2>();
    __syncthreads();  // stage `it` landed for every thread; stage it - 1 fully consumed
    if (it + NS - 1 < nst) load(it + NS - 1);
    cp_async_commit();
    const float* buf = sm_gv + (int)(it % NS) * stage_f;
    const long long v0 = vb + it * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    if (CONV) {
      // the stage in FP64, once (the previous stage's readers are past the barrier above)
      for (int f = tid; f < nv * M; f += S::NT) dbuf[f] = (double)buf[f];
      __syncthreads();
      for (int v = ph; v < nv; v += S::WPB) {
        const double* col = dbuf + v * M;
        double av[8], bv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double2 t2 = *reinterpret_cast<const double2*>(col + r0 + 2 * i);
          av[2 * i] = t2.x;
          av[2 * i + 1] = t2.y;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const double2 t2 = *reinterpret_cast<const double2*>(col + c0 + 2 * j);
          bv[2 * j] = t2.x;
          bv[2 * j + 1] = t2.y;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) accd[i][j] = fma(av[i], bv[j], accd[i][j]);
      }
      continue;
    }
    for (int v = ph; v < nv; v += S::WPB) {
      float av[8], bv[4];
      if (COL) {
#pragma unroll
        for (int i = 0; i < 8; ++i) av[i] = buf[gv_col_at(r0 + i, v)];
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = buf[gv_col_at(c0 + j, v)];
      } else {
        const float* col = buf + v * M;
        const float4 a0 = *reinterpret_cast<const float4*>(col + r0);
        const float4 a1 = *reinterpret_cast<const float4*>(col + r0 + 4);
        const float4 b = *reinterpret_cast<const float4*>(col + c0);
        av[0] = a0.x; av[1] = a0.y; av[2] = a0.z; av[3] = a0.w;
        av[4] = a1.x; av[5] = a1.y; av[6] = a1.z; av[7] = a1.w;
        bv[0] = b.x; bv[1] = b.y; bv[2] = b.z; bv[3] = b.w;
      }
      if (ACC64) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) accd[i][j] = fma((double)av[i], (double)bv[j], accd[i][j]);
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        if (++since == GV_VFLUSH) {
          since = 0;
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              accd[i][j] += (double)acc[i][j];
              acc[i][j] = 0.f;
            }
        }
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // stage buffers free: reused for the cross-warp sum
  if (!ACC64) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) accd[i][j] += (double)acc[i][j];
  }
  double* red = reinterpret_cast<double*>(sm_gv);  // [warp][32][32]
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) red[warp * 1024 + (8 * (lane >> 3) + i) * 32 + 4 * (lane & 7) + j] = accd[i][j];
  __syncthreads();
  double* dst = part + (long long)blockIdx.x * MP * MP;
  for (int e = tid; e < S::WB * 1024; e += S::NT) {
    const int b = e >> 10, rr = (e >> 5) & 31, cc = e & 31;
    double t = 0.0;
    for (int p = 0; p < S::WPB; ++p) t += red[(p * S::WB + b) * 1024 + rr * 32 + cc];
    const int R = (b == 2 ? 32 : 0) + rr, Cc = (b == 0 ? 0 : 32) + cc;
    dst[R * MP + Cc] = t;
  }
}

static int gram_mp(int M) { return M <= 16 ? 16 : M <= 32 ? 32 : M <= 48 ? 48 : M <= 64 ? 64 : 128; }

static void gram_plan(long long nvec, int* nblk, long long* vchunk) {
  const int target = 4 * num_sms();
  long long vc = ceil_div_ll(nvec, target);
  // at least 64 vectors per block: a few thousand vectors (the last unfoldings' Grams) still
  // spread over tens of blocks instead of one
  if (vc < 64) vc = 64;
  vc = ceil_div_ll(vc, 32) * 32;
  *vchunk = vc;
  *nblk = (int)std::max<long long>(1, ceil_div_ll(nvec, vc));
}

// Symmetric variant for 17 <= M <= 32 components, either layout (the exact step's Gram of a long
// unfolding with few rows; the power basis Z at widths up to 32): the upper triangle of 8 x 8
// tiles of the 32 x 32 result (10 tiles)
// times 3 vectors is 30 lanes of a warp, so a vector costs 640 FMAs instead of 1024 and a lane
// loads 16 values per 64 FMAs.  8 warps of 3 vectors take 24 vectors per step of a stage.
// FP32 products: the per-lane FP64 sums live in shared memory (row stride 65 doubles) next to
// the stages, which keeps the registers to the FP32 tile; FP64 products: in registers.
constexpr int GS_NT = 256;
constexpr int GS_LD = 65;
static size_t gram_sym_smem(int M, bool acc64, bool col) {
  const size_t stages = (col ? (size_t)32 * GV_VC : (size_t)GV_VC * M + 32) * GV_NS * sizeof(float);
  const size_t red = (size_t)GS_NT * GS_LD * sizeof(double);
  return acc64 ? std::max(stages, red) : stages + red;
}

template <bool ACC64, bool COL>
__global__ void __launch_bounds__(GS_NT, 1) k_gram_sym32(const float* __restrict__ x, long long nvec, int M,
                                                        long long ld, long long vchunk, double* __restrict__ part) {
  extern __shared__ __align__(16) float sm_gs[];
  const int stage_f = COL ? 32 * GV_VC : GV_VC * M + 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = lane % 10, u = lane / 10;  // tile, vector of the triple (u == 3: idle lanes)
  const int p = t < 4 ? 0 : t < 7 ? 1 : t < 9 ? 2 : 3;
  const int q = t < 4 ? t : t < 7 ? t - 3 : t < 9 ? t - 5 : 3;
  const long long vb = (long long)blockIdx.x * vchunk;
  const long long ve = (vb + vchunk < nvec) ? vb + vchunk : nvec;
  const long long nst = vb < ve ? (ve - vb + GV_VC - 1) / GV_VC : 0;
  auto load = [&](long long st) {
    const long long v0 = vb + st * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    float* dst = sm_gs + (int)(st % GV_NS) * stage_f;
    if (COL) {
      gv_load_col<GS_NT>(dst, x, v0, nv, M, ld, tid);
    } else {
      const int n16 = nv * M / 4;
      const float* src = x + v0 * M;
      for (int f = tid; f < n16; f += GS_NT) cp_async16(dst + 4 * f, src + 4 * f);
    }
  };
  // FP64 sums: registers (ACC64) or this thread's row of the shared block after the stages
  double* sacc = reinterpret_cast<double*>(sm_gs + GV_NS * stage_f + ((GV_NS * stage_f) & 1)) + tid * GS_LD;
  float acc[8][8];
  double accd[ACC64 ? 8 : 1][ACC64 ? 8 : 1];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[i][j] = 0.f;
      if (ACC64) accd[ACC64 ? i : 0][ACC64 ? j : 0] = 0.0;
    }
  if (!ACC64)
    for (int e = 0; e < 64; ++e) sacc[e] = 0.0;
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sacc[i * 8 + j] += (double)acc[i][j];
        acc[i][j] = 0.f;
      }
  };
  int since = 0;
#pragma unroll
  for (int st = 0; st < GV_NS - 1; ++st) {
    if (st < nst) load(st);
    cp_async_commit();
  }
  for (long long it = 0; it < nst; ++it) {
    cp_async_wait<GV_NS - 2>();
    __syncthreads();
    if (it + GV_NS - 1 < nst) load(it + GV_NS - 1);
    cp_async_commit();
    const float* buf = sm_gs + (int)(it % GV_NS) * stage_f;
    const long long v0 = vb + it * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    if (u < 3) {
      for (int v = 3 * warp + u; v < nv; v += 24) {
        float av[8], bv[8];
        if (COL) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            av[i] = buf[gv_col_at(8 * p + i, v)];
            bv[i] = buf[gv_col_at(8 * q + i, v)];
          }
        } else {
          const float* col = buf + v * M;
          const float4 a0 = *reinterpret_cast<const float4*>(col + 8 * p);
          const float4 a1 = *reinterpret_cast<const float4*>(col + 8 * p + 4);
          const float4 b0 = *reinterpret_cast<const float4*>(col + 8 * q);
          const float4 b1 = *reinterpret_cast<const float4*>(col + 8 * q + 4);
          av[0] = a0.x; av[1] = a0.y; av[2] = a0.z; av[3] = a0.w;
          av[4] = a1.x; av[5] = a1.y; av[6] = a1.z; av[7] = a1.w;
          bv[0] = b0.x; bv[1] = b0.y; bv[2] = b0.z; bv[3] = b0.w;
          bv[4] = b1.x; bv[5] = b1.y; bv[6] = b1.z; bv[7] = b1.w;
        }
        if (ACC64) {
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j)
              accd[ACC64 ? i : 0][ACC64 ? j : 0] = fma((double)av[i], (double)bv[j], accd[ACC64 ? i : 0][ACC64 ? j : 0]);
        } else {
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
          if (++since == GV_VFLUSH) {
            since = 0;
            flush();
          }
        }
      }
    }
  }
  cp_async_wait<0>();
  if (!ACC64) flush();
  __syncthreads();  // stage buffers free (ACC64 writes its sums over them)
  const double* red;  // [thread][GS_LD]
  if (ACC64) {
    double* r = reinterpret_cast<double*>(sm_gs);
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) r[tid * GS_LD + i * 8 + j] = accd[ACC64 ? i : 0][ACC64 ? j : 0];
    red = r;
  } else {
    red = sacc - tid * GS_LD;
  }
  __syncthreads();
  double* dst = part + (long long)blockIdx.x * 32 * 32;
  for (int e = tid; e < 10 * 64; e += GS_NT) {
    const int tt = e >> 6, ij = e & 63;
    double sum = 0.0;
    for (int w = 0; w < GS_NT / 32; ++w)
      for (int uu = 0; uu < 3; ++uu) sum += red[(w * 32 + uu * 10 + tt) * GS_LD + ij];
    const int pp = tt < 4 ? 0 : tt < 7 ? 1 : tt < 9 ? 2 : 3;
    const int qq = tt < 4 ? tt : tt < 7 ? tt - 3 : tt < 9 ? tt - 5 : 3;
    dst[(8 * pp + (ij >> 3)) * 32 + 8 * qq + (ij & 7)] = sum;
  }
}

// Symmetric variant with FP64 products for 33 <= M <= 48 components (the Grams of B^T and of the
// power basis Z at sketch widths 33..48), either layout: the upper triangle of TPM x TPM tiles
// of 8 x 8 (15 tiles at TPM = 5, 21 at 6) times VPW = 32 / tiles vectors per warp, FP64 sums in
// registers (a 40-wide vector costs 960 FMAs instead of the 3072 of three 32 x 32 warp blocks).
template <int TPM, bool COL>
__global__ void __launch_bounds__(GS_NT, 1) k_gram_symt(const float* __restrict__ x, long long nvec, int M,
                                                       long long ld, long long vchunk, double* __restrict__ part) {
  constexpr int MP = 8 * TPM;
  constexpr int NTILE = TPM * (TPM + 1) / 2;
  constexpr int VPW = 32 / NTILE;
  extern __shared__ __align__(16) float sm_gt[];
  const int stage_f = COL ? MP * GV_VC : GV_VC * M + MP;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = lane % NTILE, u = lane / NTILE;  // u >= VPW: idle lane
  int p = 0, rem = t;
  while (rem >= TPM - p) {
    rem -= TPM - p;
    ++p;
  }
  const int q = p + rem;
  const long long vb = (long long)blockIdx.x * vchunk;
  const long long ve = (vb + vchunk < nvec) ? vb + vchunk : nvec;
  const long long nst = vb < ve ? (ve - vb + GV_VC - 1) / GV_VC : 0;
  auto load = [&](long long st) {
    const long long v0 = vb + st * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    float* dst = sm_gt + (int)(st % GV_NS) * stage_f;
    if (COL) {
      gv_load_col<GS_NT>(dst, x, v0, nv, M, ld, tid);
    } else {
      const int n16 = nv * M / 4;
      const float* src = x + v0 * M;
      for (int f = tid; f < n16; f += GS_NT) cp_async16(dst + 4 * f, src + 4 * f);
    }
  };
  double accd[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) accd[i][j] = 0.0;
#pragma unroll
  for (int st = 0; st < GV_NS - 1; ++st) {
    if (st < nst) load(st);
    cp_async_commit();
  }
  for (long long it = 0; it < nst; ++it) {
    cp_async_wait<GV_NS - 2>();
    __syncthreads();
    if (it + GV_NS - 1 < nst) load(it + GV_NS - 1);
    cp_async_commit();
    const float* buf = sm_gt + (int)(it % GV_NS) * stage_f;
    const long long v0 = vb + it * GV_VC;
    const int nv = (int)((ve - v0 < GV_VC) ? ve - v0 : GV_VC);
    if (u < VPW) {
      for (int v = VPW * warp + u; v < nv; v += VPW * (GS_NT / 32)) {
        float av[8], bv[8];
        if (COL) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            av[i] = buf[gv_col_at(8 * p + i, v)];
            bv[i] = buf[gv_col_at(8 * q + i, v)];
          }
        } else {
          const float* col = buf + v * M;
          const float4 a0 = *reinterpret_cast<const float4*>(col + 8 * p);
          const float4 a1 = *reinterpret_cast<const float4*>(col + 8 * p + 4);
          const float4 b0 = *reinterpret_cast<const float4*>(col + 8 * q);
          const float4 b1 = *reinterpret_cast<const float4*>(col + 8 * q + 4);
          av[0] = a0.x; av[1] = a0.y; av[2] = a0.z; av[3] = a0.w;
          av[4] = a1.x; av[5] = a1.y; av[6] = a1.z; av[7] = a1.w;
          bv[0] = b0.x; bv[1] = b0.y; bv[2] = b0.z; bv[3] = b0.w;
          bv[4] = b1.x; bv[5] = b1.y; bv[6] = b1.z; bv[7] = b1.w;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) accd[i][j] = fma((double)av[i], (double)bv[j], accd[i][j]);
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();  // stage buffers free: the per-lane sums go over them
  double* red = reinterpret_cast<double*>(sm_gt);  // [thread][GS_LD]
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) red[tid * GS_LD + i * 8 + j] = accd[i][j];
  __syncthreads();
  double* dst = part + (long long)blockIdx.x * MP * MP;
  for (int e = tid; e < NTILE * 64; e += GS_NT) {
    const int tt = e >> 6, ij = e & 63;
    double sum = 0.0;
    for (int w = 0; w < GS_NT / 32; ++w)
      for (int uu = 0; uu < VPW; ++uu) sum += red[(w * 32 + uu * NTILE + tt) * GS_LD + ij];
    int pp = 0, rr = tt;
    while (rr >= TPM - pp) {
      rr -= TPM - pp;
      ++pp;
    }
    const int qq = pp + rr;
    dst[(8 * pp + (ij >> 3)) * MP + 8 * qq + (ij & 7)] = sum;
  }
}

static size_t gram_symt_smem(int MP, int M, bool col) {
  const size_t stages = (col ? (size_t)MP * GV_VC : (size_t)GV_VC * M + MP) * GV_NS * sizeof(float);
  return std::max(stages, (size_t)GS_NT * GS_LD * sizeof(double));
}

// Vector Gram (k_gram_vec): taken for 17 <= M <= 64 and enough vectors to fill the GPU, with
// x_j = x + j M (M % 4 == 0, 16-byte aligned base) or the column-major layout x[j + c es]
// (vs = 1, es >= nvec).  Returns the block size MP (0: not taken), the grid and the vectors
// per block.
static int gram_vec_plan(const float* x, long long nvec, int M, long long vs, long long es, int* grid,
                         long long* vchunk, bool* col) {
  if (M < 17 || M > 64 || nvec < 8192) return 0;
  *col = (vs == 1 && es >= nvec);
  if (!*col) {
    if (es != 1 || vs != M || (M & 3) != 0) return 0;
    if (x && (reinterpret_cast<uintptr_t>(x) & 15) != 0) return 0;
  }
  const int MP = M <= 32 ? 32 : 64;
  if (gram_vec_smem(MP, M, *col, true) > (size_t)max_optin_smem()) return 0;
  const long long g = std::min<long long>((long long)num_sms(), ceil_div_ll(nvec, 4 * GV_VC));
  long long vc = ceil_div_ll(nvec, g);
  vc = ceil_div_ll(vc, GV_VC) * GV_VC;
  *vchunk = vc;
  *grid = (int)ceil_div_ll(nvec, vc);
  return MP;
}

size_t gram_ws_bytes(long long nvec, int M) {
  int nblk;
  long long vc;
  gram_plan(nvec, &nblk, &vc);
  const int MP = gram_mp(M);
  size_t b = (size_t)nblk * MP * MP * sizeof(double);
  int g = 0;
  bool col = false;
  int MPv = gram_vec_plan(nullptr, nvec, M, M, 1, &g, &vc, &col);
  if (MPv) b = std::max(b, (size_t)g * MPv * MPv * sizeof(double));
  MPv = gram_vec_plan(nullptr, nvec, M, 1, nvec, &g, &vc, &col);
  if (MPv) b = std::max(b, (size_t)g * MPv * MPv * sizeof(double));
  return b + 4096;
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
  {
    bool col = false;
    const int MPv = gram_vec_plan(x, nvec, M, vs, es, &nblk, &vchunk, &col);
    if (MPv) {
      const size_t mk = ws.mark();
      double* part = ws.take<double>((size_t)nblk * MPv * MPv);
      if (!part) {
        set_error(TT_ERR_NOMEM, "gram workspace");
        return TT_ERR_NOMEM;
      }
      const size_t shm = gram_vec_smem(MPv, M, col, acc64);
      {
        const int mx = max_optin_smem();
#define GV_ATTR(MPV, A, C) smem_optin_k(k_gram_vec<MPV, A, C>, mx)
        GV_ATTR(32, false, false); GV_ATTR(32, true, false); GV_ATTR(64, false, false); GV_ATTR(64, true, false);
        GV_ATTR(32, false, true); GV_ATTR(32, true, true); GV_ATTR(64, false, true); GV_ATTR(64, true, true);
#undef GV_ATTR
      }
      if (MPv == 32 && gram_sym_smem(M, acc64, col) <= (size_t)max_optin_smem()) {
        {
          const int mx = max_optin_smem();
          smem_optin_k(k_gram_sym32<false, false>, mx);
          smem_optin_k(k_gram_sym32<true, false>, mx);
          smem_optin_k(k_gram_sym32<false, true>, mx);
          smem_optin_k(k_gram_sym32<true, true>, mx);
        }
        const size_t sshm = gram_sym_smem(M, acc64, col);
        const long long lds = col ? es : M;
        if (col) {
          if (acc64)
            k_gram_sym32<true, true><<<nblk, GS_NT, sshm, s>>>(x, nvec, M, lds, vchunk, part);
          else
            k_gram_sym32<false, true><<<nblk, GS_NT, sshm, s>>>(x, nvec, M, lds, vchunk, part);
        } else {
          if (acc64)
            k_gram_sym32<true, false><<<nblk, GS_NT, sshm, s>>>(x, nvec, M, lds, vchunk, part);
          else
            k_gram_sym32<false, false><<<nblk, GS_NT, sshm, s>>>(x, nvec, M, lds, vchunk, part);
        }
        count_launch();
        TT_LAUNCH_CHECK();
        launch_gram_reduce(part, nblk, 32, M, 8, w, s);
        count_launch();
        TT_LAUNCH_CHECK();
        ws.reset(mk);
        return TT_OK;
      }
      const long long ld = col ? es : M;
      if (acc64 && M > 32 && M <= 48) {
        const int MPs = M <= 40 ? 40 : 48;
        const size_t tshm = gram_symt_smem(MPs, M, col);
        if (tshm <= (size_t)max_optin_smem()) {
          {
            const int mx = max_optin_smem();
            smem_optin_k(k_gram_symt<5, false>, mx);
            smem_optin_k(k_gram_symt<5, true>, mx);
            smem_optin_k(k_gram_symt<6, false>, mx);
            smem_optin_k(k_gram_symt<6, true>, mx);
          }
          if (MPs == 40) {
            if (col)
              k_gram_symt<5, true><<<nblk, GS_NT, tshm, s>>>(x, nvec, M, ld, vchunk, part);
            else
              k_gram_symt<5, false><<<nblk, GS_NT, tshm, s>>>(x, nvec, M, ld, vchunk, part);
          } else {
            if (col)
              k_gram_symt<6, true><<<nblk, GS_NT, tshm, s>>>(x, nvec, M, ld, vchunk, part);
            else
              k_gram_symt<6, false><<<nblk, GS_NT, tshm, s>>>(x, nvec, M, ld, vchunk, part);
          }
          count_launch();
          TT_LAUNCH_CHECK();
          launch_gram_reduce(part, nblk, MPs, M, 8, w, s);
          count_launch();
          TT_LAUNCH_CHECK();
          ws.reset(mk);
          return TT_OK;
        }
      }
#define GV_LAUNCH(MPV, A, C) \
  k_gram_vec<MPV, A, C><<<nblk, GramVecShape<MPV>::NT, shm, s>>>(x, nvec, M, ld, vchunk, part)
      if (MPv == 32) {
        if (col) {
          if (acc64) GV_LAUNCH(32, true, true); else GV_LAUNCH(32, false, true);
        } else {
          if (acc64) GV_LAUNCH(32, true, false); else GV_LAUNCH(32, false, false);
        }
      } else {
        if (col) {
          if (acc64) GV_LAUNCH(64, true, true); else GV_LAUNCH(64, false, true);
        } else {
          if (acc64) GV_LAUNCH(64, true, false); else GV_LAUNCH(64, false, false);
        }
      }
#undef GV_LAUNCH
      count_launch();
      TT_LAUNCH_CHECK();
      launch_gram_reduce(part, nblk, MPv, M, 32, w, s);
      count_launch();
      TT_LAUNCH_CHECK();
      ws.reset(mk);
      return TT_OK;
    }
  }
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
  launch_gram_reduce(part, nblk, MP, M, 4, w, s);
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
// Cholesky right-looking with one barrier per column; in the trailing update thread
// (row group g, column j) loads all its rows before storing any; the pivot's reciprocal square
// root is the only special function per column.  R^-1 is formed column-parallel with no barrier
// in between: thread j back-substitutes R x = e_j (x_i = -(sum_{k>i} r_ik x_k) / r_ii), four
// partial sums per dot product.  On-chip matrices use an odd row stride (N | 1 doubles), so the
// threads of a warp, each in a different row or column, read distinct banks.
constexpr int chol_ld(int N) { return N | 1; }
__global__ void __launch_bounds__(256) k_chol_inv(const double* __restrict__ w, int N,
                                                  double* __restrict__ r_out,
                                                  double* __restrict__ rinv, double rel_tol,
                                                  int ri_smem, DevStatus* st) {
  extern __shared__ double sm[];
  const int L = chol_ld(N);
  double* A = sm;                                // N x L (row-major), upper part becomes R
  double* Ri = ri_smem ? sm + N * L : rinv;      // R^-1 column-major: stride L on chip, N in memory
  const int LR = ri_smem ? L : N;
  int* dead = reinterpret_cast<int*>(sm + (ri_smem ? 2 : 1) * N * L);
  __shared__ double dinv[128];
  __shared__ double dmax_s;
  const int tid = threadIdx.x, NT = blockDim.x;
  for (int idx = tid; idx < N * N; idx += NT) {
    const int j = idx / N, i = idx - (idx / N) * N;  // w column-major: coalesced reads
    A[i * L + j] = w[idx];
  }
  __syncthreads();
  if (tid < 32) {
    double dm = 0.0;
    for (int i = tid; i < N; i += 32) dm = fmax(dm, A[i * L + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
    if (tid == 0) dmax_s = dm;
  }
  __syncthreads();
  const double dmax = dmax_s, tol = rel_tol * dmax;
  // column j = k + 1 + (tid % CW), rows from k + 1 + tid / CW in steps of RG
  const int CW = N <= 32 ? 32 : N <= 64 ? 64 : 128;
  const int RG = NT / CW;
  for (int k = 0; k < N; ++k) {
    const double d = A[k * L + k];
    const bool live = d > tol && dmax > 0.0;
    const double rs = live ? rsqrt(d) : 0.0;  // 1 / r_kk
    if (live) {
      const double inv = rs * rs;
      const int j = k + 1 + (tid % CW);
      if (j < N) {
        const double wkj = A[k * L + j] * inv;
        const int i0 = k + 1 + tid / CW;
        constexpr int U = 8;
        for (int ib = i0; ib <= j; ib += U * RG) {
          double wk[U], wij[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int i = ib + u * RG;
            if (i <= j) {
              wk[u] = A[k * L + i];
              wij[u] = A[i * L + j];
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int i = ib + u * RG;
            if (i <= j) A[i * L + j] = fma(-wk[u], wkj, wij[u]);
          }
        }
      }
    }
    __syncthreads();
    // row k of R: A[k][c] / r_kk for c > k, r_kk = d / sqrt(d) (after the update that read it)
    for (int c = k + tid; c < N; c += NT) A[k * L + c] = live ? A[k * L + c] * rs : 0.0;
    if (tid == 0) {
      dead[k] = live ? 0 : 1;
      dinv[k] = rs;
    }
    __syncthreads();
  }
  // R out (column-major), zero below the diagonal; dead rows are zero.
  if (r_out) {
    for (int idx = tid; idx < N * N; idx += NT) {
      const int i = idx % N, j = idx / N;
      r_out[idx] = (j >= i) ? A[i * L + j] : 0.0;
    }
  }
  // R^-1, column j by thread j: x_j = 1 / r_jj, x_i = -(sum_{k=i+1..j} r_ik x_k) / r_ii.
  for (int j = tid; j < N; j += NT) {
    double* x = Ri + (long long)LR * j;
    for (int i = j + 1; i < N; ++i) x[i] = 0.0;
    if (dead[j]) {
      for (int i = 0; i <= j; ++i) x[i] = 0.0;
      continue;
    }
    x[j] = dinv[j];
    for (int i = j - 1; i >= 0; --i) {
      const double* ar = A + i * L;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int kk = i + 1;
      for (; kk + 3 <= j; kk += 4) {
        s0 = fma(ar[kk], x[kk], s0);
        s1 = fma(ar[kk + 1], x[kk + 1], s1);
        s2 = fma(ar[kk + 2], x[kk + 2], s2);
        s3 = fma(ar[kk + 3], x[kk + 3], s3);
      }
      for (; kk <= j; ++kk) s0 = fma(ar[kk], x[kk], s0);
      x[i] = -((s0 + s1) + (s2 + s3)) * dinv[i];
    }
  }
  if (ri_smem) {
    __syncthreads();
    for (int idx = tid; idx < N * N; idx += NT) {
      const int i = idx % N, j = idx / N;
      rinv[idx] = Ri[i + L * j];
    }
  }
  (void)st;
}

// Y (n x N) <- Y * T, T = R^-1 upper (FP64 in global, staged as FP32 once per block).  Blocks
// loop over tiles of 128 rows, one row per thread, outputs produced 32 columns at a time and
// written over the tile in shared memory.
template <int NP>
__global__ void __launch_bounds__(128) k_apply_rinv(float* __restrict__ y, long long n, int N,
                                                    long long vs, long long es,
                                                    const double* __restrict__ t) {
  extern __shared__ float sm_apply[];
  float* ts = sm_apply;                 // NP x NP, ts[k*NP + c]
  float* ys = ts + NP * NP;             // 128 x (NP+1): the tile, overwritten by the result
  constexpr int LD = NP + 1;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NP * NP; idx += 128) {
    const int k = idx % NP, c = idx / NP;
    ts[k * NP + c] = (k < N && c < N) ? (float)t[k + (long long)N * c] : 0.f;
  }
  // Output chunk width divides NP (NP is a multiple of 16), so cb + c < NP always.
  constexpr int CB = (NP % 32 == 0) ? 32 : 16;
  static_assert(NP % CB == 0, "chunk width must divide the padded width");
  const long long ntile = (n + 127) / 128;
  // column-major rows read / written as 16-byte runs of 4 rows
  const bool v4 = vs == 1 && es != 1 && (es & 3) == 0 && ((reinterpret_cast<uintptr_t>(y) & 15) == 0);
  for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const long long j0 = tile * 128;
    __syncthreads();  // ts ready / the previous tile's stores done
    if (es == 1) {
      for (int f = tid; f < 128 * NP; f += 128) {
        const int c = f % NP, r = f / NP;
        const long long j = j0 + r;
        ys[r * LD + c] = (j < n && c < N) ? y[j * vs + c] : 0.f;
      }
    } else if (v4) {
      // 4 consecutive rows of a column per 16-byte load; a warp covers 8 row groups x 4 columns
      for (int f = tid; f < 32 * NP; f += 128) {
        const int r4 = (f & 7) + 8 * ((f >> 5) & 3), c = ((f >> 3) & 3) + 4 * (f >> 7);
        const long long j = j0 + 4 * r4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < N) {
          if (j + 3 < n) {
            v = *reinterpret_cast<const float4*>(y + j + (long long)c * es);
          } else {
            const float* src = y + (long long)c * es;
            if (j < n) v.x = src[j];
            if (j + 1 < n) v.y = src[j + 1];
            if (j + 2 < n) v.z = src[j + 2];
          }
        }
        ys[(4 * r4) * LD + c] = v.x;
        ys[(4 * r4 + 1) * LD + c] = v.y;
        ys[(4 * r4 + 2) * LD + c] = v.z;
        ys[(4 * r4 + 3) * LD + c] = v.w;
      }
    } else {
      for (int f = tid; f < 128 * NP; f += 128) {
        const int r = f % 128, c = f / 128;
        const long long j = j0 + r;
        ys[r * LD + c] = (j < n && c < N) ? y[j * vs + (long long)c * es] : 0.f;
      }
    }
    __syncthreads();
    // Row tid in place: T is upper triangular, so output columns cb.. need inputs k < cb + CB
    // only; chunks run from the last one down and overwrite inputs no later chunk reads.
    for (int cb = NP - CB; cb >= 0; cb -= CB) {
      float outv[CB];
#pragma unroll
      for (int c = 0; c < CB; ++c) outv[c] = 0.f;
      for (int k = 0; k < cb + CB; ++k) {
        const float yk = ys[tid * LD + k];
#pragma unroll
        for (int c = 0; c < CB; ++c) outv[c] = fmaf(yk, ts[k * NP + cb + c], outv[c]);
      }
#pragma unroll
      for (int c = 0; c < CB; ++c) ys[tid * LD + cb + c] = outv[c];
    }
    __syncthreads();
    if (es == 1) {
      for (int f = tid; f < 128 * NP; f += 128) {
        const int c = f % NP, r = f / NP;
        const long long j = j0 + r;
        if (j < n && c < N) y[j * vs + c] = ys[r * LD + c];
      }
    } else if (v4) {
      for (int f = tid; f < 32 * NP; f += 128) {
        const int r4 = (f & 7) + 8 * ((f >> 5) & 3), c = ((f >> 3) & 3) + 4 * (f >> 7);
        const long long j = j0 + 4 * r4;
        if (c >= N || j >= n) continue;
        const float4 v = make_float4(ys[(4 * r4) * LD + c], ys[(4 * r4 + 1) * LD + c], ys[(4 * r4 + 2) * LD + c],
                                     ys[(4 * r4 + 3) * LD + c]);
        float* dst = y + (long long)c * es;
        if (j + 3 < n) {
          *reinterpret_cast<float4*>(dst + j) = v;
        } else {
          dst[j] = v.x;
          if (j + 1 < n) dst[j + 1] = v.y;
          if (j + 2 < n) dst[j + 2] = v.z;
        }
      }
    } else {
      for (int f = tid; f < 128 * NP; f += 128) {
        const int r = f % 128, c = f / 128;
        const long long j = j0 + r;
        if (j < n && c < N) y[j * vs + (long long)c * es] = ys[r * LD + c];
      }
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

// Cluster helpers: rank in the cluster, cluster size, cluster-wide barrier (release / acquire),
// and an FP64 load from the same shared-memory offset in another CTA of the cluster.
__device__ __forceinline__ unsigned cl_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cl_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cl_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ double ld_peer_f64(const double* p, unsigned rank) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  unsigned ra;
  double v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
  return v;
}

// CholeskyQR2 of an n x N sketch (N <= 64) in one launch: a cluster of up to 8 CTAs, each
// holding `rpc` consecutive rows in shared memory (64 < N <= 80: one CTA of 256 threads, the
// Gram summed straight into W, no R output).  Y is staged row-major with a padded
// stride S (S/4 odd, so the float4 row accesses of neighbouring threads fall in distinct
// banks); per pass:
//   each CTA's partial Gram Y_c^T Y_c in FP64 (4x4 register tiles over the upper tile
//   triangle, row groups reduced through shared memory), summed over the cluster through
//   distributed shared memory in rank order (every CTA gets the same bits, so the redundant
//   factorisations agree), right-looking Cholesky in FP64 (one barrier per column, dead
//   pivots below rel_tol * max diag), then Q = Y R^-1 by forward substitution, one row per
//   thread in FP32 registers against an FP32 copy of R (column-major, diagonal stored as
//   1/r_cc).
// Optional R output (column-major) = R2 * R1, written by rank 0.  Each pass has its own partial
// buffer, so a CTA that runs ahead never overwrites a partial a peer is still reading; the
// final cluster barrier keeps every CTA's shared memory alive until the peers are done.
template <int NP>
__global__ void __launch_bounds__(NP > 64 ? 256 : 512) k_cholqr2_small(float* __restrict__ y, int n, int N,
                                                                      long long vs, long long es, int S,
                                                                      int rpc, double* __restrict__ r,
                                                                      double rel_tol) {
  constexpr int NT = NP > 64 ? 256 : 512;  // the wide rows of the substitution need the registers
  extern __shared__ __align__(16) unsigned char sm_cq[];
  const unsigned crank = cl_rank(), csize = cl_size();
  const int row0 = (int)crank * rpc;
  const int nl = max(0, min(rpc, n - row0));                         // rows of this CTA
  const int WN = (N * N + 1) & ~1;
  float* Ys = reinterpret_cast<float*>(sm_cq);                       // rpc x S
  double* Wp = reinterpret_cast<double*>(Ys + (size_t)rpc * S);      // 2 x N x N partials
  double* W = NP > 64 ? Wp : Wp + 2 * WN;                            // N x N row-major
  float* Rf = reinterpret_cast<float*>(W + WN);                      // NP x NP, Rf[c*NP+k] = R[k][c]
  float* invd = Rf + NP * NP;                                        // NP
  double* R1 = reinterpret_cast<double*>(invd + NP);                 // N x N (only with r)
  const int tid = threadIdx.x;
  const int TTa = (N + 3) >> 2;
  const int ngrp = S >> 2;
  for (int f = tid; f < nl * ngrp; f += NT) {
    const int i = f % nl, q4 = f / nl;
    const long long gi = row0 + i;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int c = 4 * q4 + e;
      v[e] = (c < N) ? y[gi * vs + (long long)c * es] : 0.f;
    }
    *reinterpret_cast<float4*>(&Ys[(size_t)i * S + 4 * q4]) = make_float4(v[0], v[1], v[2], v[3]);
  }
  // Tile assignment for the Gram: tile t of the TTa x TTa upper triangle, row group g.
  const int nt = TTa * (TTa + 1) / 2;
  const int groups = min(32, max(1, NT / nt));
  const int t = tid % nt, g = tid / nt;
  const bool act = g < groups;
  int ta = 0, rem = act ? t : 0;
  while (rem >= TTa - ta) {
    rem -= TTa - ta;
    ++ta;
  }
  const int tb = ta + rem;
  for (int pass = 0; pass < 2; ++pass) {
    double* Wq = NP > 64 ? W : Wp + pass * WN;
    __syncthreads();
    double acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0.0;
    if (act) {
      for (int v = g; v < nl; v += groups) {
        const float4 xa = *reinterpret_cast<const float4*>(&Ys[(size_t)v * S + 4 * ta]);
        const float4 xb = *reinterpret_cast<const float4*>(&Ys[(size_t)v * S + 4 * tb]);
        const double av[4] = {xa.x, xa.y, xa.z, xa.w};
        const double bv[4] = {xb.x, xb.y, xb.z, xb.w};
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p * 4 + q] = fma(av[p], bv[q], acc[p * 4 + q]);
      }
    }
    for (int gg = 0; gg < groups; ++gg) {
      if (act && g == gg) {
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int i = 4 * ta + p, j = 4 * tb + q;
            if (i < N && j < N) Wq[i * N + j] = (gg == 0 ? 0.0 : Wq[i * N + j]) + acc[p * 4 + q];
          }
      }
      __syncthreads();
    }
    // Sum the partials over the cluster (upper triangle), in rank order.
    cl_sync();
    for (int idx = tid; idx < N * N; idx += NT) {
      const int i = idx / N, j = idx - (idx / N) * N;
      if (i > j) continue;
      double a = Wq[idx];
      if (csize > 1) {
        a = 0.0;
        for (unsigned q = 0; q < csize; ++q) a += ld_peer_f64(Wq + idx, q);
      }
      W[idx] = a;
    }
    __syncthreads();
    double dmax = 0.0;
    for (int k = 0; k < N; ++k) dmax = fmax(dmax, W[k * N + k]);
    const double tol = rel_tol * dmax;
    __syncthreads();  // every thread has read the diagonal before the first update changes it
    for (int k = 0; k < N; ++k) {
      const double d = W[k * N + k];
      if (d > tol && dmax > 0.0) {
        // trailing update of the upper triangle: thread (row group tid / CW, column tid % CW);
        // a thread's rows in chunks of 8, each chunk loaded before any of it is stored
        constexpr int CW = NP > 64 ? 128 : 64, RG = NT / CW;
        const double inv = 1.0 / d;
        const int j = k + 1 + (tid % CW);
        if (j < N) {
          const double wkj = W[k * N + j] * inv;
          for (int i0 = k + 1 + tid / CW; i0 <= j; i0 += 8 * RG) {
            double wk[8], wij[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int i = i0 + RG * u;
              if (i <= j) {
                wk[u] = W[k * N + i];
                wij[u] = W[i * N + j];
              }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int i = i0 + RG * u;
              if (i <= j) W[i * N + j] = fma(-wk[u], wkj, wij[u]);
            }
          }
        }
      }
      __syncthreads();
    }
    // R[k][c] = W[k][c] / sqrt(W[k][k]) on live rows (c >= k); dead rows are zero.
    for (int idx = tid; idx < NP * NP; idx += NT) {
      const int c = idx / NP, k = idx % NP;
      float v = 0.f;
      if (c < N && k < c) {
        const double d = W[k * N + k];
        if (d > tol && dmax > 0.0) v = (float)(W[k * N + c] / sqrt(d));
      }
      Rf[idx] = v;
    }
    for (int c = tid; c < NP; c += NT) {
      float v = 0.f;
      if (c < N) {
        const double d = W[c * N + c];
        if (d > tol && dmax > 0.0) v = (float)(1.0 / sqrt(d));
      }
      invd[c] = v;
    }
    if (r) {
      for (int idx = tid; idx < N * N; idx += NT) {
        const int k = idx % N, c = idx / N;  // column-major (k, c)
        const double dk = W[k * N + k];
        const bool live = dk > tol && dmax > 0.0;
        if (pass == 0) {
          R1[idx] = (live && c >= k) ? W[k * N + c] / sqrt(dk) : 0.0;
        } else {
          double a = 0.0;
          if (live && c >= k) {
            const double sk = 1.0 / sqrt(dk);
            for (int j = k; j <= c; ++j) a += W[k * N + j] * sk * R1[j + N * c];
          }
          if (crank == 0) r[idx] = a;
        }
      }
    }
    __syncthreads();
    // Forward substitution q R = y, one row per thread.
    for (int i = tid; i < nl; i += NT) {
      float q[NP];
#pragma unroll
      for (int j4 = 0; j4 < NP / 4; ++j4) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j4 < TTa) v = *reinterpret_cast<const float4*>(&Ys[(size_t)i * S + 4 * j4]);
        q[4 * j4] = v.x;
        q[4 * j4 + 1] = v.y;
        q[4 * j4 + 2] = v.z;
        q[4 * j4 + 3] = v.w;
      }
#pragma unroll
      for (int c = 0; c < NP; ++c) {
        // four independent partial sums (one per float4 lane) shorten the dependency chain
        float a0 = q[c], a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
        for (int k4 = 0; k4 < (c + 3) / 4; ++k4) {
          const float4 rr = *reinterpret_cast<const float4*>(&Rf[c * NP + 4 * k4]);
          a0 = fmaf(-q[4 * k4], rr.x, a0);
          a1 = fmaf(-q[4 * k4 + 1], rr.y, a1);
          a2 = fmaf(-q[4 * k4 + 2], rr.z, a2);
          a3 = fmaf(-q[4 * k4 + 3], rr.w, a3);
        }
        q[c] = ((a0 + a1) + (a2 + a3)) * invd[c];
      }
      if (pass == 0) {
#pragma unroll
        for (int j4 = 0; j4 < NP / 4; ++j4)
          if (j4 < TTa)
            *reinterpret_cast<float4*>(&Ys[(size_t)i * S + 4 * j4]) =
                make_float4(q[4 * j4], q[4 * j4 + 1], q[4 * j4 + 2], q[4 * j4 + 3]);
      } else {
        const long long gi = row0 + i;
#pragma unroll
        for (int c = 0; c < NP; ++c)
          if (c < N) y[gi * vs + (long long)c * es] = q[c];
      }
    }
  }
  cl_sync();  // peers may still be reading this CTA's second partial
}

static int max_optin_smem() { return dev_smem_max(); }

// Cluster shape and shared-memory bytes of k_cholqr2_small: the fewest CTAs (at most 8) with
// at least 128 rows each that fit in shared memory; 0 when the sketch does not fit.
static size_t cholqr2_small_smem(long long n, int N, bool want_r, int* S_out, int* cl_out, int* rpc_out) {
  if (N < 1 || N > 80 || n < 1 || n > (1LL << 20)) return 0;
  if (N > 64 && want_r) return 0;  // the one-CTA wide variant forms no R
  const int NP = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : N <= 64 ? 64 : 80;
  int S = 4 * ((N + 3) / 4);
  if (((S / 4) & 1) == 0) S += 4;
  const size_t WN = ((size_t)N * N + 1) & ~(size_t)1;
  const size_t fixed = (NP > 64 ? 1 : 3) * WN * 8 + (size_t)NP * NP * 4 + NP * 4 + (want_r ? (size_t)N * N * 8 : 0);
  const int cl_max = NP > 64 ? 1 : 8;
  for (int cl = (int)std::min<long long>(cl_max, std::max<long long>(1, (n + 127) / 128)); cl <= cl_max; ++cl) {
    const long long rpc = (n + cl - 1) / cl;
    const size_t bytes = (size_t)rpc * S * 4 + fixed;
    if (bytes <= (size_t)max_optin_smem()) {
      *S_out = S;
      *cl_out = cl;
      *rpc_out = (int)rpc;
      return bytes;
    }
  }
  return 0;
}

static int cholqr_passes(float* y, long long n, int N, long long vs, long long es, double* r, Arena& ws,
                         DevStatus* st, cudaStream_t s, int passes, bool acc64);

int launch_cholqr2(float* y, long long n, int N, long long vs, long long es, double* r,
                   Arena& ws, DevStatus* st, cudaStream_t s) {
  return cholqr_passes(y, n, N, vs, es, r, ws, st, s, 2, true);
}

// One CholeskyQR pass: the orthonormalisation between power iterations, which only has to keep
// the basis well conditioned (the sketch that follows is orthonormalised by CholeskyQR2).  The
// Gram is FP32-accumulated (FP64 across chunks of vectors), or FP64 per product with acc64: a
// basis whose columns span a graded spectrum (condition kappa) then comes out with
// orthogonality ~kappa * 2^-24, still well conditioned, where the FP32 Gram (condition
// kappa^2) would lose the small directions.
int launch_orth_power(float* y, long long n, int N, long long vs, long long es, Arena& ws, DevStatus* st,
                      cudaStream_t s, bool acc64) {
  return cholqr_passes(y, n, N, vs, es, nullptr, ws, st, s, 1, acc64);
}

static int cholqr_passes(float* y, long long n, int N, long long vs, long long es, double* r, Arena& ws,
                         DevStatus* st, cudaStream_t s, int passes, bool acc64) {
  if (N <= 0 || n <= 0) return TT_OK;
  if (N > TT_MAX_SMALL) {
    set_error(TT_ERR_UNSUPPORTED, "cholqr2 width %d > %d", N, TT_MAX_SMALL);
    return TT_ERR_UNSUPPORTED;
  }
  int S = 0, cl = 1, rpc = 0;
  const size_t sshm = cholqr2_small_smem(n, N, r != nullptr, &S, &cl, &rpc);
  if (sshm > 0) {
    {
      const int mx = max_optin_smem();
      smem_optin_k(k_cholqr2_small<16>, mx);
      smem_optin_k(k_cholqr2_small<32>, mx);
      smem_optin_k(k_cholqr2_small<48>, mx);
      smem_optin_k(k_cholqr2_small<64>, mx);
      smem_optin_k(k_cholqr2_small<80>, mx);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl, 1, 1);
    cfg.blockDim = dim3(N > 64 ? 256 : 512, 1, 1);
    cfg.dynamicSmemBytes = sshm;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const int nn = (int)n;
    const double tol = 1e-12;
    cudaError_t e;
    if (N <= 16)
      e = cudaLaunchKernelEx(&cfg, k_cholqr2_small<16>, y, nn, N, vs, es, S, rpc, r, tol);
    else if (N <= 32)
      e = cudaLaunchKernelEx(&cfg, k_cholqr2_small<32>, y, nn, N, vs, es, S, rpc, r, tol);
    else if (N <= 48)
      e = cudaLaunchKernelEx(&cfg, k_cholqr2_small<48>, y, nn, N, vs, es, S, rpc, r, tol);
    else if (N <= 64)
      e = cudaLaunchKernelEx(&cfg, k_cholqr2_small<64>, y, nn, N, vs, es, S, rpc, r, tol);
    else
      e = cudaLaunchKernelEx(&cfg, k_cholqr2_small<80>, y, nn, N, vs, es, S, rpc, r, tol);
    if (e == cudaSuccess) {
      count_launch();
      TT_LAUNCH_CHECK();
      return TT_OK;
    }
    // A cluster that cannot be placed (its CTAs' shared memory on one GPC) falls through to the
    // multi-launch path below.
    (void)cudaGetLastError();
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
  const int ri_smem = 2 * (size_t)N * chol_ld(N) * sizeof(double) + N * sizeof(int) + 16 <= 200 * 1024;
  const size_t shm = (size_t)(ri_smem ? 2 : 1) * N * chol_ld(N) * sizeof(double) + N * sizeof(int) + 16;
  smem_optin_k(k_chol_inv, 200 * 1024);
  smem_optin_k(k_apply_rinv<16>, 200 * 1024);
  smem_optin_k(k_apply_rinv<32>, 200 * 1024);
  smem_optin_k(k_apply_rinv<48>, 200 * 1024);
  smem_optin_k(k_apply_rinv<64>, 200 * 1024);
  smem_optin_k(k_apply_rinv<128>, 200 * 1024);
  for (int pass = 0; pass < passes; ++pass) {
    TT_TRY(launch_gram(y, n, N, vs, es, w, acc64, ws, s));
    k_chol_inv<<<1, 256, shm, s>>>(w, N, pass == 0 ? r1 : r2, rinv, 1e-12, ri_smem, st);
    count_launch();
    TT_LAUNCH_CHECK();
    const size_t ashm = ((size_t)NP * NP + 128 * (size_t)(NP + 1)) * sizeof(float);
    // persistent blocks (R^-1 staged once per block), as many as fit on the SMs
    const int per_sm = std::max(1, std::min(8, (int)((200u * 1024u) / (ashm + 1024))));
    const int grid = (int)std::min<long long>(ceil_div_ll(n, 128), (long long)per_sm * num_sms());
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
  if (r && passes == 2) {
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
// Single-matrix solver for N <= 64 (bl_solver.cuh): one CTA of bl_shape's warp count, compiled
// for the smallest thread bound that holds it, so that the compiler may give each thread the
// registers it needs (at 1024 threads it has 64 and spills): V is row-resident up to N = 46
// (at most 8 warps for N <= 32, 12 for N <= 46); 46 < N <= 64 splits V and takes 1024 threads.
template <int MAXT, int VN>
__global__ void __launch_bounds__(MAXT, 1) k_syev_bl(const double* __restrict__ w_in, int N,
                                                   double* __restrict__ evals,
                                                   double* __restrict__ evecs, int max_sweeps,
                                                   DevStatus* st) {
  extern __shared__ __align__(16) double sm_bl[];
  const int sw = bl_solve<VN>(w_in, N, evals, evecs, max_sweeps, sm_bl);
  if (threadIdx.x == 0 && st) {
    atomicMax(&st->sweeps, min(sw, max_sweeps));
    if (sw > max_sweeps) dev_fail(st, TT_ERR_NOCONV, max_sweeps);
  }
}

// Large-N variant (64 < N <= 128) of the Brent-Luk solver.  W alone stays in shared memory: its
// upper triangle packed by rows (row P stored from column P & ~1, so every 2 x 2 block row is a
// 16-byte load), double-buffered (2 x 66.5 KB for N = 128).  The eigenvectors are not updated
// round by round: the rotation warps log each round's renormalised FP64 (c, s) pairs to global
// memory (so the replay's per-round chain has no conversion or renormalisation), and
// k_bl_replay applies them afterwards to the rows of V, one CTA per row (rows are independent),
// with the same moves.  Two warps compute the next round's rotations during the update; every
// W thread's block addresses and the rotation lanes' entry offsets are computed once.
__device__ __forceinline__ int blp_off(int P, int Np) {
  // sum over rows p < P of (Np - (p & ~1)): pairs of rows (2a, 2a + 1) hold 2 (Np - 2a) entries
  const int a = P >> 1;
  return 2 * (a * Np - a * (a - 1)) + (P & 1) * (Np - 2 * a);
}

__global__ void __launch_bounds__(1024) k_syev_blw(const double* __restrict__ w_in, int N,
                                                    double* __restrict__ evals, double2* __restrict__ tlog,
                                                    int* __restrict__ meta, int max_sweeps, DevStatus* st) {
  constexpr int RW0 = 30;  // warps 30, 31 compute the next round's rotations
  constexpr int NE = RW0 * 32;
  extern __shared__ __align__(16) double sm_blw[];
  const int Np = N + (N & 1);
  const int NR = Np - 1;
  const int H = Np / 2;
  const int PS = blp_off(Np, Np);
  double* Wb0 = sm_blw;
  double* Wb1 = Wb0 + PS;
  __shared__ double2 pcs[2][64];
  __shared__ int mv[128], imv[128];
  __shared__ double dg[128];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // offset of entry (P, Q), P <= Q: arithmetic (a few integer ops) rather than a table lookup,
  // which would add a shared-memory load to every access
  auto at = [&](int P, int Q) { return blp_off(P, Np) + (Q - (P & ~1)); };
  for (int P = tid; P < Np; P += blockDim.x) {
    const int x = P % 2 == 0 ? P / 2 : Np - 1 - P / 2;
    const int xn = x == 0 ? 0 : (x == 1 ? NR : x - 1);
    const int Pn = bl_pos(xn, Np);
    mv[P] = Pn;
    imv[Pn] = P;
  }
  __syncthreads();
  for (int e = tid; e < 2 * PS; e += blockDim.x) Wb0[e] = 0.0;
  __syncthreads();
  for (int idx = tid; idx < Np * Np; idx += blockDim.x) {
    const int i = idx / Np, j = idx - (idx / Np) * Np;
    const int Pi = bl_pos(i, Np), Pj = bl_pos(j, Np);
    if (Pi > Pj) continue;
    double v = 0.0;
    if (i < N && j < N) v = 0.5 * (w_in[i + (long long)N * j] + w_in[j + (long long)N * i]);
    Wb0[at(Pi, Pj)] = v;
  }
  double dm = 0.0;
  for (int i = 0; i < N; ++i) dm = fmax(dm, fabs(w_in[i + (long long)N * i]));
  const double inv_s = dm > 0.0 ? 1.0 / dm : 1.0;
  __syncthreads();
  const int rl = tid - NE;  // rotation lane (0..63) on the rotation warps
  if (warp >= RW0 && rl < H) {
    const int k = rl;
    const int i0 = k, i1 = Np - 1 - k;
    float2 r = make_float2(1.0f, 0.0f);
    if (i0 < N && i1 < N)
      r = jacobi_cs32(Wb0[at(2 * k, 2 * k)], Wb0[at(2 * k + 1, 2 * k + 1)], Wb0[at(2 * k, 2 * k + 1)], inv_s);
    double c, sn;
    rot_from_cs32(r, c, sn);
    pcs[0][k] = make_double2(c, sn);
    tlog[k] = make_double2(c, sn);
  }
  __syncthreads();
  const int NWB = H * (H + 1) / 2;
  constexpr int MAXIT = (64 * 65 / 2 + NE - 1) / NE;
  // per block of this thread: the pair indices (a | b << 8, -1 for none), the offsets of its two
  // rows in W and of its four entries' next-round upper positions (fixed over the rounds)
  int dsc[MAXIT], ldo[MAXIT], sto[MAXIT][4];
#pragma unroll
  for (int u = 0; u < MAXIT; ++u) {
    const int it = tid + u * NE;
    dsc[u] = -1;
    ldo[u] = 0;
    sto[u][0] = sto[u][1] = sto[u][2] = sto[u][3] = 0;
    if (warp < RW0 && it < NWB) {
      int a = 0, rem = it;
      while (rem >= H - a) {
        rem -= H - a;
        ++a;
      }
      const int b = a + rem;
      dsc[u] = a | (b << 8);
      ldo[u] = at(2 * a, 2 * b);
      const int r0 = mv[2 * a], r1 = mv[2 * a + 1], q0 = mv[2 * b], q1 = mv[2 * b + 1];
      sto[u][0] = at(min(r0, q0), max(r0, q0));
      sto[u][1] = at(min(r0, q1), max(r0, q1));
      sto[u][2] = at(min(r1, q0), max(r1, q0));
      sto[u][3] = at(min(r1, q1), max(r1, q1));
    }
  }
  int aP = 0, xP = 0, aQ = 0, xQ = 0;
  int wo[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // offsets of the entries the rotation lane reads
  if (warp >= RW0 && rl < H) {
    const int P = imv[2 * rl], Q = imv[2 * rl + 1];
    aP = P >> 1;
    xP = P & 1;
    aQ = Q >> 1;
    xQ = Q & 1;
    const int P0 = 2 * aP, Q0 = 2 * aQ;
    auto ou = [&](int r, int c2) { return at(min(r, c2), max(r, c2)); };
    wo[0] = ou(P0, P0);
    wo[1] = ou(P0, P0 + 1);
    wo[2] = ou(P0 + 1, P0 + 1);
    wo[3] = ou(Q0, Q0);
    wo[4] = ou(Q0, Q0 + 1);
    wo[5] = ou(Q0 + 1, Q0 + 1);
    wo[6] = ou(P0, Q0);
    wo[7] = ou(P0 + 1, Q0);
    wo[8] = ou(P0, Q0 + 1);
    wo[9] = ou(P0 + 1, Q0 + 1);
  }
  int R = 0;
  int sweep = 0;
  bool converged = false;
  for (; sweep < max_sweeps; ++sweep) {
    bool stop = false;
    for (int rnd = 0; rnd < NR; ++rnd, ++R) {
      const int cb = R & 1;
      const double* W = cb ? Wb1 : Wb0;
      double* Wn = cb ? Wb0 : Wb1;
      const double2* cs_ = pcs[cb];
      if (warp < RW0) {
#pragma unroll
        for (int u = 0; u < MAXIT; ++u) {
          const int dd = dsc[u];
          if (dd < 0) continue;
          const int a = dd & 255, b = (dd >> 8) & 255;
          const double2 csa = cs_[a], csb = cs_[b];
          const double ca = csa.x, sa = csa.y, cbv = csb.x, sb = csb.y;
          // row 2a + 1 starts (Np - 2a) entries after row 2a (both stored from column 2a)
          const double2 r0v = *reinterpret_cast<const double2*>(&W[ldo[u]]);
          const double2 r1v = *reinterpret_cast<const double2*>(&W[ldo[u] + (Np - 2 * a)]);
          const double w00 = r0v.x, w01 = r0v.y, w11 = r1v.y;
          const double w10 = (a == b) ? w01 : r1v.x;
          const double x00 = ca * w00 - sa * w10, x01 = ca * w01 - sa * w11;
          const double x10 = sa * w00 + ca * w10, x11 = sa * w01 + ca * w11;
          const double y00 = x00 * cbv - x01 * sb, y01 = x00 * sb + x01 * cbv;
          const double y10 = x10 * cbv - x11 * sb, y11 = x10 * sb + x11 * cbv;
          Wn[sto[u][0]] = y00;
          Wn[sto[u][1]] = y01;
          if (a != b) Wn[sto[u][2]] = y10;
          Wn[sto[u][3]] = y11;
        }
      } else if (rl < H) {
        const int rn = (rnd + 1 == NR) ? 0 : rnd + 1;
        bool live = true;
        if (Np != N) {
          const int xs = bl_slot(Np - 1, rn, NR);
          live = (xs != rl) && (xs != Np - 1 - rl);
        }
        float2 r = make_float2(1.0f, 0.0f);
        if (live) {
          const double cP = cs_[aP].x, sP = cs_[aP].y, cQ = cs_[aQ].x, sQ = cs_[aQ].y;
          const double tP0 = xP ? sP : cP, tP1 = xP ? cP : -sP;
          const double tQ0 = xQ ? sQ : cQ, tQ1 = xQ ? cQ : -sQ;
          const double p0 = tP0 * W[wo[0]] + tP1 * W[wo[1]];
          const double p1 = tP0 * W[wo[1]] + tP1 * W[wo[2]];
          const double q0 = tQ0 * W[wo[3]] + tQ1 * W[wo[4]];
          const double q1 = tQ0 * W[wo[4]] + tQ1 * W[wo[5]];
          const double m0 = tP0 * W[wo[6]] + tP1 * W[wo[7]];
          const double m1 = tP0 * W[wo[8]] + tP1 * W[wo[9]];
          r = jacobi_cs32(p0 * tP0 + p1 * tP1, q0 * tQ0 + q1 * tQ1, m0 * tQ0 + m1 * tQ1, inv_s);
        }
        double c, sn;
        rot_from_cs32(r, c, sn);
        pcs[cb ^ 1][rl] = make_double2(c, sn);
        tlog[(size_t)(R + 1) * H + rl] = make_double2(c, sn);  // rotations of round R + 1
      }
      __syncthreads();
      if (rnd + 1 == NR) {
        int need = 0;
        for (int idx = tid; idx < Np * Np; idx += blockDim.x) {
          const int P = idx / Np, Q = idx - (idx / Np) * Np;
          if (P < Q && jacobi_needed(Wn[at(P, P)], Wn[at(Q, Q)], Wn[at(P, Q)], inv_s)) need = 1;
        }
        if (!__syncthreads_or(need)) stop = true;
      }
    }
    if (stop) {
      converged = true;
      ++sweep;
      break;
    }
  }
  // eigenvalues by rank; meta = [rounds, rank of index 0..N-1, final position of index 0..N-1]
  const double* Wf = (R & 1) ? Wb1 : Wb0;
  if (tid < N) {
    const int P = bl_pos(bl_slot(tid, R, NR), Np);
    dg[tid] = Wf[at(P, P)];
  }
  __syncthreads();
  if (tid < N) {
    double la = dg[tid];
    if (la != la) la = -INFINITY;
    int rank = 0;
    for (int b = 0; b < N; ++b) {
      double lb = dg[b];
      if (lb != lb) lb = -INFINITY;
      rank += (lb > la || (lb == la && b < tid)) ? 1 : 0;
    }
    evals[rank] = dg[tid];
    meta[1 + tid] = rank;
    meta[1 + 128 + tid] = bl_pos(bl_slot(tid, R, NR), Np);
  }
  if (tid == 0) {
    meta[0] = R;
    if (st) {
      atomicMax(&st->sweeps, sweep);
      if (!converged) dev_fail(st, TT_ERR_NOCONV, sweep);
    }
  }
}

// Replays the logged rotations on row i of V (one CTA per row, one thread per pair; V starts as
// the identity with index i at its round-0 position) and writes the eigenvectors by rank.
__global__ void __launch_bounds__(64) k_bl_replay(const double2* __restrict__ tlog, const int* __restrict__ meta,
                                                  int N, double* __restrict__ evecs) {
  __shared__ double vb[2][128];
  __shared__ int mvs[128];
  const int Np = N + (N & 1), H = Np / 2, NR = Np - 1;
  const int i = blockIdx.x, k = threadIdx.x;
  for (int P = k; P < Np; P += blockDim.x) {
    const int x = P % 2 == 0 ? P / 2 : Np - 1 - P / 2;
    const int xn = x == 0 ? 0 : (x == 1 ? NR : x - 1);
    mvs[P] = bl_pos(xn, Np);
    vb[0][P] = (P == bl_pos(i, Np)) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int rounds = meta[0];
  const int m0 = k < H ? mvs[2 * k] : 0, m1 = k < H ? mvs[2 * k + 1] : 0;
  constexpr int U = 8;
  for (int R0 = 0; R0 < rounds; R0 += U) {
    double2 tf[U];
#pragma unroll
    for (int j = 0; j < U; ++j)
      tf[j] = (k < H && R0 + j < rounds) ? tlog[(size_t)(R0 + j) * H + k] : make_double2(1.0, 0.0);
#pragma unroll
    for (int j = 0; j < U; ++j) {
      if (R0 + j >= rounds) break;
      const int cb = (R0 + j) & 1;
      if (k < H) {
        const double c = tf[j].x, sn = tf[j].y;
        const double v0 = vb[cb][2 * k], v1 = vb[cb][2 * k + 1];
        vb[cb ^ 1][m0] = v0 * c - v1 * sn;
        vb[cb ^ 1][m1] = v0 * sn + v1 * c;
      }
      __syncthreads();
    }
  }
  const double* vf = vb[rounds & 1];
  for (int a = k; a < N; a += blockDim.x) evecs[i + (long long)N * meta[1 + a]] = vf[meta[1 + 128 + a]];
}

size_t syev_ws_bytes(int N, int max_sweeps) {
  if (N <= 64) return 0;
  const int Np = N + (N & 1);
  const int sw = max_sweeps > 0 ? max_sweeps : 40;
  return ((size_t)sw * (Np - 1) + 2) * (Np / 2) * sizeof(double2) + (1 + 2 * 128) * sizeof(int) + 1024;
}

int launch_syev(const double* w, int N, double* evals, double* evecs, int max_sweeps, Arena& ws,
                DevStatus* st, cudaStream_t s) {
  if (N <= 0) return TT_OK;
  if (N > TT_MAX_SMALL) {
    set_error(TT_ERR_UNSUPPORTED, "eigen-solver size %d > %d", N, TT_MAX_SMALL);
    return TT_ERR_UNSUPPORTED;
  }
  if (N <= 64) {
    const int Nps = N + (N & 1);
    const size_t shm_bl = 2 * (size_t)Nps * Nps * sizeof(double);
    int iso, warps;
    bl_shape(N, N <= 46, &iso, &warps);
    if (N <= 32) {
      smem_optin_k(k_syev_bl<256, 32>, shm_bl);
      k_syev_bl<256, 32><<<1, 32 * warps, shm_bl, s>>>(w, N, evals, evecs, max_sweeps, st);
    } else if (N <= 46) {
      smem_optin_k(k_syev_bl<384, 48>, shm_bl);
      k_syev_bl<384, 48><<<1, 32 * warps, shm_bl, s>>>(w, N, evals, evecs, max_sweeps, st);
    } else {
      smem_optin_k(k_syev_bl<1024, 0>, shm_bl);
      k_syev_bl<1024, 0><<<1, 32 * warps, shm_bl, s>>>(w, N, evals, evecs, max_sweeps, st);
    }
    count_launch();
    TT_LAUNCH_CHECK();
    return TT_OK;
  }
  // 64 < N <= 128: packed Brent-Luk on W, eigenvectors by replaying the logged rotations
  const int Np = N + (N & 1), H = Np / 2;
  const int sw = max_sweeps > 0 ? max_sweeps : 40;
  const size_t mk = ws.mark();
  double2* tlog = ws.take<double2>(((size_t)sw * (Np - 1) + 2) * H);
  int* meta = ws.take<int>(1 + 2 * 128);
  if (!tlog || !meta) {
    set_error(TT_ERR_NOMEM, "eigen-solver rotation log");
    return TT_ERR_NOMEM;
  }
  const size_t shm = 2 * (size_t)(2 * (H * Np - H * (H - 1))) * sizeof(double);
  TT_TRY(smem_optin_k(k_syev_blw, shm));
  k_syev_blw<<<1, 1024, shm, s>>>(w, N, evals, tlog, meta, sw, st);
  count_launch();
  TT_LAUNCH_CHECK();
  k_bl_replay<<<N, 64, 0, s>>>(tlog, meta, N, evecs);
  count_launch();
  TT_LAUNCH_CHECK();
  ws.reset(mk);
  return TT_OK;
}

// ---------------------------------------------------------------------------------------
// Leading eigenpairs of a symmetric positive semidefinite W (64 < N <= 128) for steps that use
// only the first few: orthogonal (subspace) iteration on a block of kSubDim columns, then
// Rayleigh-Ritz.  One CTA holds W (FP64) and two N x kSubDim blocks in shared memory (column-major,
// column stride NP = N rounded up to even, the pad row zero).  The start block is Philox
// Gaussian; every second multiplication by W the block is orthonormalised by one CholeskyQR pass
// (FP64 Gram by a warp per entry, right-looking Cholesky, forward substitution with each row in
// registers), and the last basis gets a second pass (CholeskyQR2).  The projected matrix
// H = Y^T W Y (kSubDim x kSubDim) goes to the N <= 32 Jacobi solver and the Ritz vectors are Y
// times its eigenvectors.  The span of the first k Ritz vectors converges to W's leading
// k-dimensional invariant subspace as (lambda_{kSubDim+1} / lambda_k)^kSubMults.
// ---------------------------------------------------------------------------------------
constexpr int kSubDim = 32;
constexpr int kSubMults = 16;

// Y = an orthonormal basis of span(Y), in place.  Columns whose pivot is below 1e-28 of the
// largest diagonal of Y^T Y (directions W annihilates) come out zero.
__device__ void sub_cholqr(double* Y, int NP, double* G, double* rf) {
  constexpr int B = kSubDim;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int e = warp; e < B * (B + 1) / 2; e += nw) {
    int p = 0, rem = e;
    while (rem >= B - p) {
      rem -= B - p;
      ++p;
    }
    const int q = p + rem;
    double acc = 0.0;
    for (int i = lane; i < NP; i += 32) acc = fma(Y[p * NP + i], Y[q * NP + i], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      G[p * B + q] = acc;
      G[q * B + p] = acc;
    }
  }
  __syncthreads();
  double dmax = 0.0;
  for (int i = 0; i < B; ++i) dmax = fmax(dmax, G[i * B + i]);
  const double tol = 1e-28 * dmax;
  __syncthreads();  // every thread has read the diagonal before the first update changes it
  // right-looking Cholesky on the upper triangle (row kk is final after step kk)
  for (int kk = 0; kk < B; ++kk) {
    const double dk = G[kk * B + kk];
    if (dk > tol && dmax > 0.0) {
      const int j = kk + 1 + lane;
      if (j < B) {
        const double wkj = G[kk * B + j] / dk;
        for (int i = kk + 1 + warp; i <= j; i += nw) G[i * B + j] -= G[kk * B + i] * wkj;
      }
    }
    __syncthreads();
  }
  // rf[kk B + c] = R[kk][c] (kk < c, live pivots), rf[B B + c] = 1 / R[c][c] (0: dead column)
  for (int idx = tid; idx < B * B + B; idx += blockDim.x) {
    if (idx < B * B) {
      const int kk = idx / B, c = idx - kk * B;
      const double dk = G[kk * B + kk];
      rf[idx] = (kk < c && dk > tol && dmax > 0.0) ? G[kk * B + c] / sqrt(dk) : 0.0;
    } else {
      const double dc = G[(idx - B * B) * (B + 1)];
      rf[idx] = (dc > tol && dmax > 0.0) ? 1.0 / sqrt(dc) : 0.0;
    }
  }
  __syncthreads();
  for (int i = tid; i < NP; i += blockDim.x) {  // row i: y R = z (forward substitution)
    double y[B];
#pragma unroll
    for (int c = 0; c < B; ++c) {
      double a0 = Y[c * NP + i], a1 = 0.0;
#pragma unroll
      for (int kk = 0; kk < c; ++kk) {
        if (kk & 1) a1 = fma(-y[kk], rf[kk * B + c], a1);
        else a0 = fma(-y[kk], rf[kk * B + c], a0);
      }
      y[c] = (a0 + a1) * rf[B * B + c];
    }
#pragma unroll
    for (int c = 0; c < B; ++c) Y[c * NP + i] = y[c];
  }
  __syncthreads();
}

// Z = W Y (NP x kSubDim): thread (i, g) computes rows i and i + NP/2 for columns 8g .. 8g + 7,
// two k at a time (Y's column pairs as 16-byte broadcasts, W's rows read as its columns).
__device__ void sub_mult(const double* __restrict__ W, const double* __restrict__ Y, double* __restrict__ Z,
                         int NP) {
  const int H = NP / 2, tid = threadIdx.x;
  if (tid < 4 * H) {
    const int i = tid % H, g = tid / H;
    double a0[8], a1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a0[j] = a1[j] = 0.0;
    const double* y0 = Y + (size_t)(8 * g) * NP;
    for (int k = 0; k < NP; k += 2) {
      const double w00 = W[k * NP + i], w01 = W[(k + 1) * NP + i];
      const double w10 = W[k * NP + i + H], w11 = W[(k + 1) * NP + i + H];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 y = *reinterpret_cast<const double2*>(y0 + j * NP + k);
        a0[j] = fma(w01, y.y, fma(w00, y.x, a0[j]));
        a1[j] = fma(w11, y.y, fma(w10, y.x, a1[j]));
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      Z[(8 * g + j) * NP + i] = a0[j];
      Z[(8 * g + j) * NP + i + H] = a1[j];
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(512, 1) k_subspace_iter(const double* __restrict__ w_in, int N,
                                                           unsigned long long seed, double* __restrict__ y_out,
                                                           double* __restrict__ h_out) {
  extern __shared__ __align__(16) double sm_sub[];
  constexpr int B = kSubDim;
  const int NP = N + (N & 1);
  double* Ws = sm_sub;           // NP x NP
  double* Ys = Ws + NP * NP;     // NP x B
  double* Zs = Ys + NP * B;      // NP x B
  double* G = Zs + NP * B;       // B x B
  double* rf = G + B * B;        // B x B + B
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < NP * NP; idx += blockDim.x) {
    const int i = idx % NP, k = idx / NP;
    Ws[idx] = (i < N && k < N) ? 0.5 * (w_in[i + (long long)N * k] + w_in[k + (long long)N * i]) : 0.0;
  }
  for (int q = tid; q < NP * (B / 4); q += blockDim.x) {
    const int i = q % NP, c4 = 4 * (q / NP);
    const float4 g = philox_normal4((unsigned long long)q, 0x5ab5u, seed);
    const bool live = i < N;
    Ys[(c4 + 0) * NP + i] = live ? g.x : 0.0;
    Ys[(c4 + 1) * NP + i] = live ? g.y : 0.0;
    Ys[(c4 + 2) * NP + i] = live ? g.z : 0.0;
    Ys[(c4 + 3) * NP + i] = live ? g.w : 0.0;
  }
  __syncthreads();
  sub_cholqr(Ys, NP, G, rf);
  for (int it = 0; it < kSubMults / 2; ++it) {
    sub_mult(Ws, Ys, Zs, NP);
    sub_mult(Ws, Zs, Ys, NP);
    sub_cholqr(Ys, NP, G, rf);
  }
  sub_cholqr(Ys, NP, G, rf);
  sub_mult(Ws, Ys, Zs, NP);
  // H = Y^T Z symmetrised (a warp per entry), Y out column-major N x B
  for (int e = warp; e < B * (B + 1) / 2; e += nw) {
    int p = 0, rem = e;
    while (rem >= B - p) {
      rem -= B - p;
      ++p;
    }
    const int q = p + rem;
    double a = 0.0;
    for (int i = lane; i < NP; i += 32)
      a = fma(Ys[p * NP + i], Zs[q * NP + i], fma(Ys[q * NP + i], Zs[p * NP + i], a));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) {
      h_out[p + B * q] = 0.5 * a;
      h_out[q + B * p] = 0.5 * a;
    }
  }
  for (int idx = tid; idx < N * B; idx += blockDim.x) {
    const int i = idx % N, c = idx / N;
    y_out[idx] = Ys[c * NP + i];
  }
}

// evecs (N x N) = [Y E, 0], evals = [lambda(H), 0]: the kSubDim Ritz pairs, zero beyond them.
__global__ void k_ritz(const double* __restrict__ y, const double* __restrict__ eh, const double* __restrict__ lh,
                       int N, double* __restrict__ evals, double* __restrict__ evecs) {
  constexpr int B = kSubDim;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < (long long)N * N;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % N), j = (int)(idx / N);
    double v = 0.0;
    if (j < B)
      for (int c = 0; c < B; ++c) v = fma(y[i + (long long)N * c], eh[c + B * j], v);
    evecs[idx] = v;
    if (i == 0) evals[j] = j < B ? lh[j] : 0.0;
  }
}

size_t syev_top_smem(int N) {
  const size_t np = (size_t)(N + (N & 1));
  return (np * np + 2 * np * kSubDim + 2 * (size_t)kSubDim * kSubDim + kSubDim) * sizeof(double);
}

int launch_syev_top(const double* w, int N, double* evals, double* evecs, int max_sweeps, Arena& ws,
                    DevStatus* st, cudaStream_t s) {
  if (N <= 64 || N > TT_MAX_SMALL) return launch_syev(w, N, evals, evecs, max_sweeps, ws, st, s);
  const size_t mk = ws.mark();
  double* y = ws.take<double>((size_t)N * kSubDim);
  double* h = ws.take<double>((size_t)kSubDim * kSubDim);
  double* eh = ws.take<double>((size_t)kSubDim * kSubDim);
  double* lh = ws.take<double>(kSubDim);
  if (!y || !h || !eh || !lh) {
    set_error(TT_ERR_NOMEM, "subspace eigen-solver workspace");
    return TT_ERR_NOMEM;
  }
  const size_t shm = syev_top_smem(N);
  TT_TRY(smem_optin_k(k_subspace_iter, shm));
  k_subspace_iter<<<1, 512, shm, s>>>(w, N, 0x7c3a9e15ull, y, h);
  count_launch();
  TT_LAUNCH_CHECK();
  TT_TRY(launch_syev(h, kSubDim, lh, eh, max_sweeps, ws, st, s));
  k_ritz<<<ceil_div(N * N, 256), 256, 0, s>>>(y, eh, lh, N, evals, evecs);
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

// out (Rout, cols) <- in (Rin, cols), rows Rin..Rout-1 zero (Rin <= Rout), column-major.
__global__ void k_expand_rows(const float* __restrict__ in, int Rin, float* __restrict__ out, int Rout,
                              long long cols) {
  const long long total = (long long)Rout * cols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long c = idx / Rout;
    const int a = (int)(idx - c * Rout);
    out[idx] = (a < Rin) ? in[a + (long long)Rin * c] : 0.f;
  }
}

int launch_expand_rows(const float* in, int Rin, float* out, int Rout, long long cols, cudaStream_t s) {
  const long long total = (long long)Rout * cols;
  if (total <= 0) return TT_OK;
  k_expand_rows<<<(int)std::min<long long>(ceil_div_ll(total, 256), 8LL * num_sms()), 256, 0, s>>>(
      in, Rin, out, Rout, cols);
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

// Residual energies of the probe columns outside range(Q): out[j] = ||y_j - Q (Q^T y_j)||^2,
// Q (m x ks, FP32, ldq, orthonormal columns), Y0 (m x q, FP64, ldy).  One block per probe
// column; FP64 throughout, so the difference of two nearly equal energies is not formed.
__global__ void __launch_bounds__(256) k_probe_resid(const float* __restrict__ q, long long m, int ks, long long ldq,
                                                     const double* __restrict__ y0, long long ldy,
                                                     double* __restrict__ out) {
  extern __shared__ double sh_pr[];  // c[ks] + 8 warp partials
  double* c = sh_pr;
  double* red = sh_pr + ks;
  const int j = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* y = y0 + (long long)j * ldy;
  // c = Q^T y: warp w takes columns w, w + 8, ...
  for (int a = warp; a < ks; a += 8) {
    const float* qa = q + (long long)a * ldq;
    double t = 0.0;
    for (long long i = lane; i < m; i += 32) t = fma((double)qa[i], y[i], t);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) c[a] = t;
  }
  __syncthreads();
  double acc = 0.0;
  for (long long i = tid; i < m; i += blockDim.x) {
    double r = y[i];
    for (int a = 0; a < ks; ++a) r = fma(-(double)q[i + (long long)a * ldq], c[a], r);
    acc = fma(r, r, acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    out[j] = t;
  }
}

int launch_probe_resid(const float* q, long long m, int ks, long long ldq, const double* y0, long long ldy, int nq,
                       double* out, cudaStream_t s) {
  if (nq <= 0) return TT_OK;
  const size_t shm = (size_t)(ks + 8) * sizeof(double);
  k_probe_resid<<<nq, 256, shm, s>>>(q, m, ks, ldq, y0, ldy, out);
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
  TT_TRY(smem_optin_k(k_recon_err, 200 * 1024));
  const int grid = (int)std::min<long long>(ceil_div_ll(N, 32), 8LL * num_sms());
  k_recon_err<<<grid, 256, shm, s>>>(x, n1, N, g1, r0, r1, mrg, acc);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

}  // namespace ttr
