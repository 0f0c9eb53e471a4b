// tcgen05 / TMA tensor-core engine for the two bulk GEMMs of the TT/TR-SVD chain (sm_100a).
//
//   projection  out[j, c] = sum_k A[k + m j] Q[k + ldq c]   (A^T Q; K-major A and Q)
//   sketch      Y[i, c]   = sum_j A[i + m j] W[j + ldw c]   (A W;   MN-major A, K-major W)
//
// Both read the FP32 unfolding straight from HBM with TMA into 128B-swizzled shared memory
// and feed kind::tf32 MMAs (FP32 accumulation in TMEM); no conversion pass over A exists.
// Every operand goes through a TFLOAT32 tensor map: the TMA unit then rounds FP32 to TF32 to
// nearest on the way into shared memory.  Operands loaded as plain FP32 are truncated toward
// zero by the MMA, which biases every product by about -3e-4 (measured); rounding removes the
// bias, and the projection additionally splits Q into hi + lo parts.
// Warp roles per CTA (192 threads): warp 0 = TMA producer, warp 1 = TMEM owner and MMA
// issuer (one thread), warps 2-5 = epilogue (TMEM -> registers -> global).  Every mbarrier
// wait is bounded by a wall-clock limit; a role that gives up raises a shared abort flag
// and a TT_ERR_TIMEOUT device status, and the CTA drains its own TMA copies and MMAs
// before releasing TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdlib.h>

#include <algorithm>

#include "kernels.cuh"

namespace ttr {
namespace {

// Wall-clock limit of every pipeline wait (settable per device, tt_ctx_set_wait_limit), and the
// fixed limit of the waits that drain a CTA's own copies after a failure: those always get the
// full 2 s, so lowering the pipeline limit never lets a CTA leave with copies in flight.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
__device__ unsigned long long g_wait_limit_ns = kWaitLimitNs;

// ---------------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the phase of parity `parity` to complete.  Returns false when the time
// limit passes or another role raised the abort flag.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer() - t0 > g_wait_limit_ns) return false;
  }
}
// Bounded pipeline wait without an abort flag (the per-warp pipelines of the exact Gram).
__device__ __forceinline__ bool mbar_wait_limit(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer(), lim = g_wait_limit_ns;
  while (!mbar_try_wait(bar, parity))
    if (globaltimer() - t0 > lim) return false;
  return true;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = globaltimer();
  while (!mbar_try_wait(bar, parity))
    if (globaltimer() - t0 > kWaitLimitNs) return false;
  return true;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"((unsigned long long)map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"((unsigned long long)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
// 32 lanes x 16 columns of 32-bit accumulators; registers valid after tmem_wait_ld().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
// Named barrier among `nthreads` threads that also ORs a predicate across them, so every
// participant takes the same branch afterwards.
__device__ __forceinline__ bool named_bar_or(uint32_t id, uint32_t nthreads, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n barrier.red.or.pred q, %2, %3, p;\n"
      " selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptors (sm_100 format: version 1 at bit 46, layout at 61-63).
// K-major, swizzle `mode` (2 = 128B, 4 = 64B, 6 = 32B); SBO = stride of 8-row groups.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t mode, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46) | ((uint64_t)mode << 61);
}
// MN-major, 128B swizzle with 32B atoms (the tf32 MN-major layout): LBO = stride between
// 32-element MN blocks, SBO = stride between 4-row K groups.
__device__ __forceinline__ uint64_t desc_mn_sw128_32b(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46) | ((uint64_t)1u << 61);
}
// Instruction descriptor of kind::tf32 with FP32 accumulation.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int a_mn_major, int b_mn_major) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn_major << 15) |
         ((uint32_t)b_mn_major << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__host__ __device__ constexpr uint32_t pow2_cols(uint32_t c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

// Barrier block at the end of the stage ring.
struct Bars {
  uint32_t base;
  int stages;
  __device__ uint32_t full(int s) const { return base + 8u * s; }
  __device__ uint32_t empty(int s) const { return base + 8u * (stages + s); }
  __device__ uint32_t tfull(int b) const { return base + 8u * (2 * stages + b); }       // b < 4
  __device__ uint32_t tempty(int b) const { return base + 8u * (2 * stages + 4 + b); }  // b < 4
  __device__ uint32_t drain() const { return base + 8u * (2 * stages + 8); }
  __host__ __device__ static constexpr int count(int stages) { return 2 * stages + 9; }
};

// Wait (bounded) until the most recent TMA fill of every stage has landed; fill number f used
// stage f % stages with phase parity (f / stages) & 1.  Called by a producer that stopped
// early, so no later fill can complete the same parity again.
__device__ __forceinline__ void drain_fills(const Bars& bars, int stages, long long nissued) {
  for (int s = 0; s < stages; ++s) {
    if (nissued <= s) break;
    const long long last = s + (long long)stages * ((nissued - 1 - s) / stages);
    mbar_wait_bounded(bars.full(s), (uint32_t)((last / stages) & 1));
  }
}

// ---------------------------------------------------------------------------------------
// projection kernel: out = A^T Q   (persistent over 128-column tiles of A)
// ---------------------------------------------------------------------------------------
// SPLIT: Q arrives as an exactly-TF32 high part (tmB) and its FP32 remainder (tmB2); each
// K-step issues A*Qhi and A*Qlo into the same accumulator, so Q carries FP32 precision.
template <int BN, int STAGES, bool SPLIT>
__global__ void __launch_bounds__(320, 1)
    k_project_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmB2, long long n, int N, int KB,
                 float* __restrict__ out, long long ldo, int mode, int r0, int r1, DevStatus* st) {
  constexpr int BM = 128;
  constexpr uint32_t A_BYTES = BM * 128;
  constexpr uint32_t B_BYTES = BN * 128;
  constexpr uint32_t STAGE_BYTES = A_BYTES + (SPLIT ? 2 : 1) * B_BYTES;  // 1 KB aligned
  constexpr uint32_t BNP = pow2_cols(BN);
  constexpr uint32_t TMEM_COLS = pow2_cols(4 * BNP);  // four accumulators, two per epilogue group
  constexpr uint32_t IDESC = idesc_tf32(BM, BN, 0, 0);
  static_assert(STAGE_BYTES % 1024 == 0, "stage alignment");

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* barmem = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barmem + Bars::count(STAGES));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const Bars bars{smem_u32(barmem), STAGES};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntiles = (n + BM - 1) / BM;
  const uint32_t sbase = smem_u32(smem);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(bars.full(s), 1);
      mbar_init(bars.empty(s), 1);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(bars.tfull(b), 1);
      mbar_init(bars.tempty(b), 4);
    }
    mbar_init(bars.drain(), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmB) : "memory");
    if (SPLIT) asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmB2) : "memory");
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      long long nissued = 0;  // stage fills issued so far (drain bookkeeping)
      bool ok = true;
      for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int j0 = (int)(tile * BM);
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.empty(stage), phase ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          mbar_expect_tx(bars.full(stage), STAGE_BYTES);
          const uint32_t sa = sbase + stage * STAGE_BYTES;
          tma_load_2d(sa, &tmA, bars.full(stage), kb * 32, j0);
          tma_load_2d(sa + A_BYTES, &tmB, bars.full(stage), kb * 32, 0);
          if (SPLIT) tma_load_2d(sa + A_BYTES + B_BYTES, &tmB2, bars.full(stage), kb * 32, 0);
          ++nissued;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 1);
        // drain: every issued copy must land before the CTA can leave
        drain_fills(bars, STAGES, nissued);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int t = 0;
      for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++t) {
        const int buf = t & 3;
        const uint32_t tph = (uint32_t)((t >> 2) & 1);
        if (!mbar_wait(bars.tempty(buf), tph ^ 1u, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + (uint32_t)buf * BNP;
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.full(stage), phase, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = sbase + stage * STAGE_BYTES;
          const uint64_t da = desc_kmajor(sa, 2, 1024);
          const uint64_t db = desc_kmajor(sa + A_BYTES, 2, 1024);
          const uint64_t db2 = desc_kmajor(sa + A_BYTES + B_BYTES, 2, 1024);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            mma_tf32(d, da + 2ull * s, db + 2ull * s, IDESC, (kb | s) ? 1u : 0u);
            if (SPLIT) mma_tf32(d, da + 2ull * s, db2 + 2ull * s, IDESC, 1u);
          }
          mma_commit(bars.empty(stage));
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(bars.tfull(buf));
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 2);
      }
      mma_commit(bars.drain());
      mbar_wait_bounded(bars.drain(), 0);
    }
  } else {
    // Two epilogue groups of four warps (one per TMEM lane quadrant each) take alternate tiles:
    // group e drains accumulators e and e + 2, so up to four tiles are in flight.
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    const int e = (warp - 2) >> 2;
    int t = e;
    const bool vec = (mode == OUT_ROWMAJOR) && ((ldo & 3) == 0) && ((N & 3) == 0) &&
                     ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    for (long long tile = blockIdx.x + (long long)e * gridDim.x; tile < ntiles; tile += 2LL * gridDim.x, t += 2) {
      const int buf = t & 3;
      const uint32_t tph = (uint32_t)((t >> 2) & 1);
      if (!mbar_wait(bars.tfull(buf), tph, abort_flag)) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 3);
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)buf * BNP;
      uint32_t r[BN];
#pragma unroll
      for (int c = 0; c < BN; c += 16) tmem_ld16(taddr + c, &r[c]);
      tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < BN; ++c) asm volatile("" : "+r"(r[c])::"memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bars.tempty(buf));
      const long long j = tile * BM + q * 32 + lane;
      if (BN <= 32 && mode == OUT_PERM231) {  // the launcher sends the bond permute only for BN <= 32
        // Bond permute through shared memory: for each a, the warp's 32 columns j form one
        // contiguous run of r1 * 32 outputs (b fastest), written with coalesced stores.
        float* stg = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(barmem) + 256) + (warp - 2) * 32 * (BN + 1);
#pragma unroll
        for (int c = 0; c < BN; ++c) stg[lane * (BN + 1) + c] = __uint_as_float(r[c]);
        __syncwarp();
        const long long jw = tile * BM + q * 32;
        const int nj = (int)((n - jw) < 32 ? (n - jw) : 32);
        if ((r1 & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
          // lane = column j: its r1 outputs of bond index a are contiguous (b fastest), so each
          // lane stores them as float4s and a warp store covers 32 consecutive 16-byte chunks
          if (lane < nj) {
            const float* sr = stg + lane * (BN + 1);
            for (int ai = 0; ai < r0; ++ai) {
              float* dst = out + (long long)r1 * (jw + lane + n * (long long)ai);
              for (int bi = 0; bi < r1; bi += 4)
                *reinterpret_cast<float4*>(dst + bi) =
                    make_float4(sr[ai + r0 * bi], sr[ai + r0 * (bi + 1)], sr[ai + r0 * (bi + 2)],
                                sr[ai + r0 * (bi + 3)]);
            }
          }
        } else {
          for (int ai = 0; ai < r0; ++ai) {
            float* dst = out + (long long)r1 * (jw + n * (long long)ai);
            for (int f = lane; f < r1 * nj; f += 32) {
              const int jl = f / r1, bi = f - jl * r1;
              dst[f] = stg[jl * (BN + 1) + ai + r0 * bi];
            }
          }
        }
        __syncwarp();
      } else if (j < n) {
        if (mode == OUT_ROWMAJOR) {
          float* o = out + j * ldo;
          if (vec) {
#pragma unroll
            for (int c = 0; c < BN; c += 4)
              if (c < N)
                *reinterpret_cast<float4*>(o + c) =
                    make_float4(__uint_as_float(r[c]), __uint_as_float(r[c + 1]),
                                __uint_as_float(r[c + 2]), __uint_as_float(r[c + 3]));
          } else {
#pragma unroll
            for (int c = 0; c < BN; ++c)
              if (c < N) o[c] = __uint_as_float(r[c]);
          }
        } else {  // OUT_COLMAJOR
#pragma unroll
          for (int c = 0; c < BN; ++c)
            if (c < N) out[j + ldo * (long long)c] = __uint_as_float(r[c]);
        }
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------------------
// sketch kernel: Y = A W, split over the long dimension n; MT 128-row accumulators per CTA
// share each W tile.  A is MN-major (rows contiguous), W K-major (column-major n x N).
// ---------------------------------------------------------------------------------------
template <int BN, int MT, int BK, int STAGES>
__global__ void __launch_bounds__(192, 1)
    k_sketch_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                long long m, long long n, int N, long long kchunk, int nsplit, int ngroups,
                double* __restrict__ part, DevStatus* st, int a3d) {
  constexpr int BLK = MT * 4;                   // 32-row blocks per group
  constexpr uint32_t ABLK = BK * 128;           // one 32-row block, BK columns
  constexpr uint32_t A_BYTES = BLK * ABLK;
  constexpr uint32_t B_BYTES = BN * BK * 4;
  constexpr uint32_t STAGE_BYTES = (A_BYTES + B_BYTES + 1023) & ~1023u;
  constexpr uint32_t BNP = (BN + 15) / 16 * 16;
  constexpr uint32_t TMEM_COLS = pow2_cols(MT * BNP);
  constexpr uint32_t IDESC = idesc_tf32(128, BN, 1, 0);
  constexpr uint32_t BSW = BK == 8 ? 6u : BK == 16 ? 4u : 2u;  // 32B / 64B / 128B swizzle
  constexpr uint32_t BSBO = 8 * BK * 4;
  static_assert(MT * BNP <= 512, "TMEM capacity");
  static_assert(BK == 8 || BK == 16 || BK == 32, "BK");

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* barmem = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barmem + Bars::count(STAGES));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const Bars bars{smem_u32(barmem), STAGES};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int units = ngroups * nsplit;
  const uint32_t sbase = smem_u32(smem);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(bars.full(s), 1);
      mbar_init(bars.empty(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bars.tfull(b), 1);
      mbar_init(bars.tempty(b), 4);
    }
    mbar_init(bars.drain(), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmB) : "memory");
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      long long nissued = 0;  // stage fills issued so far (drain bookkeeping)
      bool ok = true;
      for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
        const int g = u % ngroups, sp = u / ngroups;
        const int i0 = g * MT * 128;
        const long long jb = (long long)sp * kchunk;
        const long long je = (jb + kchunk < n) ? jb + kchunk : n;
        const int KB = (int)((je - jb + BK - 1) / BK);
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.empty(stage), phase ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          mbar_expect_tx(bars.full(stage), A_BYTES + B_BYTES);
          const uint32_t sa = sbase + stage * STAGE_BYTES;
          const int jc = (int)(jb + (long long)kb * BK);
          if (a3d) {
            // all BLK 32-row blocks of the group in one copy: (row in block, column, block)
            tma_load_3d(sa, &tmA, bars.full(stage), 0, jc, i0 / 32);
          } else {
#pragma unroll 1
            for (int blk = 0; blk < BLK; ++blk)
              tma_load_2d(sa + blk * ABLK, &tmA, bars.full(stage), i0 + blk * 32, jc);
          }
          tma_load_2d(sa + A_BYTES, &tmB, bars.full(stage), jc, 0);
          ++nissued;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 11);
        drain_fills(bars, STAGES, nissued);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int t = 0;
      for (int u = blockIdx.x; u < units && ok; u += gridDim.x, ++t) {
        const int sp = u / ngroups;
        const long long jb = (long long)sp * kchunk;
        const long long je = (jb + kchunk < n) ? jb + kchunk : n;
        const int KB = (int)((je - jb + BK - 1) / BK);
        if (!mbar_wait(bars.tempty(0), (uint32_t)(t & 1) ^ 1u, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.full(stage), phase, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = sbase + stage * STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < BK / 8; ++ks) {
            const uint64_t db = desc_kmajor(sa + A_BYTES + ks * 32, BSW, BSBO);
#pragma unroll
            for (int tt = 0; tt < MT; ++tt) {
              const uint64_t da = desc_mn_sw128_32b(sa + (4 * tt) * ABLK + ks * 1024, ABLK, 512);
              mma_tf32(tmem_base + tt * BNP, da, db, IDESC, (kb | ks) ? 1u : 0u);
            }
          }
          mma_commit(bars.empty(stage));
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(bars.tfull(0));
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 12);
      }
      mma_commit(bars.drain());
      mbar_wait_bounded(bars.drain(), 0);
    }
  } else {
    const int q = warp & 3;
    int t = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++t) {
      const int g = u % ngroups, sp = u / ngroups;
      if (!mbar_wait(bars.tfull(0), (uint32_t)(t & 1), abort_flag)) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 13);
        break;
      }
      tc_fence_after();
      for (int tt = 0; tt < MT; ++tt) {
        const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + tt * BNP;
        uint32_t r[BN];
#pragma unroll
        for (int c = 0; c < BN; c += 16) tmem_ld16(taddr + c, &r[c]);
        tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < BN; ++c) asm volatile("" : "+r"(r[c])::"memory");
        const long long i = (long long)g * MT * 128 + tt * 128 + q * 32 + lane;
        if (i < m) {
          double* dst = part + (long long)sp * N * m + i;
#pragma unroll
          for (int c = 0; c < BN; ++c)
            if (c < N) dst[(long long)c * m] = (double)__uint_as_float(r[c]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bars.tempty(0));
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------------------
// Gram kernel: W = A A^T for an m-row unfolding (m <= 128), split over the columns.
// The 128-row MMA operand is either the unfolding viewed with 128/m consecutive columns
// stacked (grouped view, 128 % m == 0: the diagonal m x m blocks of the 128 x 128 product are
// the Gram contributions) or the m rows padded with zero rows by the TMA (padded view).
// Both MMA operands are the same MN-major shared-memory tile.
// ---------------------------------------------------------------------------------------
template <int NB, int STAGES>
__global__ void __launch_bounds__(192, 1)
    k_gram_tc(const __grid_constant__ CUtensorMap tmA, long long ncols, int m, int grouped,
              long long kchunk, int nsplit, double* __restrict__ part, DevStatus* st) {
  constexpr int BK = 32;
  constexpr uint32_t ABLK = BK * 128;           // one 32-row block, BK columns
  constexpr uint32_t STAGE_BYTES = 4 * ABLK;    // 128 rows
  constexpr uint32_t NBP = pow2_cols(NB);
  constexpr uint32_t TMEM_COLS = pow2_cols(2 * NBP);  // two accumulators: MMA fills one while the epilogue drains the other
  constexpr uint32_t IDESC = idesc_tf32(128, NB, 1, 1);

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* barmem = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(barmem + Bars::count(STAGES));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  float* gsum = reinterpret_cast<float*>(tmem_slot + 4);  // per-CTA Gram accumulator, m x (m+1) used
  const Bars bars{smem_u32(barmem), STAGES};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t sbase = smem_u32(smem);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(bars.full(s), 1);
      mbar_init(bars.empty(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bars.tfull(b), 1);
      mbar_init(bars.tempty(b), 4);
    }
    mbar_init(bars.drain(), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmA) : "memory");
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      long long nissued = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nsplit && ok; u += gridDim.x) {
        const long long jb = (long long)u * kchunk;
        const long long je = (jb + kchunk < ncols) ? jb + kchunk : ncols;
        const int KB = (int)((je - jb + BK - 1) / BK);
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.empty(stage), phase ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          mbar_expect_tx(bars.full(stage), STAGE_BYTES);
          const uint32_t sa = sbase + stage * STAGE_BYTES;
          const int jc = (int)(jb + (long long)kb * BK);
#pragma unroll
          for (int blk = 0; blk < 4; ++blk) tma_load_2d(sa + blk * ABLK, &tmA, bars.full(stage), blk * 32, jc);
          ++nissued;
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 21);
        drain_fills(bars, STAGES, nissued);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int t = 0;
      for (int u = blockIdx.x; u < nsplit && ok; u += gridDim.x, ++t) {
        const long long jb = (long long)u * kchunk;
        const long long je = (jb + kchunk < ncols) ? jb + kchunk : ncols;
        const int KB = (int)((je - jb + BK - 1) / BK);
        const int buf = t & 1;
        if (!mbar_wait(bars.tempty(buf), (uint32_t)((t >> 1) & 1) ^ 1u, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dacc = tmem_base + (uint32_t)buf * NBP;
        for (int kb = 0; kb < KB; ++kb) {
          if (!mbar_wait(bars.full(stage), phase, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = sbase + stage * STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < BK / 8; ++ks) {
            const uint64_t da = desc_mn_sw128_32b(sa + ks * 1024, ABLK, 512);
            mma_tf32(dacc, da, da, IDESC, (kb | ks) ? 1u : 0u);
          }
          mma_commit(bars.empty(stage));
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(bars.tfull(buf));
      }
      if (!ok) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 22);
      }
      mma_commit(bars.drain());
      mbar_wait_bounded(bars.drain(), 0);
    }
  } else {
    const int et = threadIdx.x - 64;           // 0..127
    const int q = warp & 3;
    const int row = q * 32 + lane;             // row of the 128-row operand
    int t = 0;
    for (int u = blockIdx.x; u < nsplit; u += gridDim.x, ++t) {
      for (int idx = et; idx < m * m; idx += 128) gsum[(idx / m) * (m + 1) + idx % m] = 0.f;
      const int buf = t & 1;
      const bool ok = mbar_wait(bars.tfull(buf), (uint32_t)((t >> 1) & 1), abort_flag);
      // all four epilogue warps leave together if any of them gave up
      if (named_bar_or(1, 128, !ok)) {
        *abort_flag = 1;
        dev_fail(st, TT_ERR_TIMEOUT, 23);
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)buf * NBP;
      uint32_t r[NB];
#pragma unroll
      for (int c = 0; c < NB; c += 16) tmem_ld16(taddr + c, &r[c]);
      tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < NB; ++c) asm volatile("" : "+r"(r[c])::"memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bars.tempty(buf));
      // Gram row (row % m) gets columns [blk*m, blk*m + m) of its diagonal block.
      const int gi = grouped ? row % m : row;
      const int c0 = grouped ? (row / m) * m : 0;
      if (gi < m && c0 + m <= NB) {
#pragma unroll
        for (int c = 0; c < NB; ++c) {
          if (c >= c0 && c < c0 + m) atomicAdd(&gsum[gi * (m + 1) + (c - c0)], __uint_as_float(r[c]));
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      double* dst = part + (long long)u * m * m;
      for (int idx = et; idx < m * m; idx += 128) dst[idx] = (double)gsum[(idx % m) * (m + 1) + idx / m];
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------------------
// Exact Gram of short vectors on the CUDA cores: W = sum_j x_j x_j^T, x_j = M <= 32
// contiguous floats (the exact step's Gram of an unfolding with at most 32 rows, e.g. the
// 32 x 33,554,432 first unfolding of a 32^6 tensor; largeMatrixSelfMulti_once_device,
// ttdec6_singleGPU.cu:388-401, which the reference runs on FP16 tensor cores).
//
// The tensor cores cannot serve this Gram: their FP32 accumulator truncates, which biases a
// long sum by ~1e-7 of its leading entries, while the smallest kept eigenvalue of such an
// unfolding can sit at 1e-5 of the largest.  Here the products are FP32 (round to nearest)
// and go through FP32 partial sums of 64 vectors into FP64 sums, so every rounding error is
// unbiased and the result is accurate to ~1e-9 relative.
//
// Each warp runs its own TMA pipeline: 48-vector boxes (6 KB, 128B-swizzled rows) through 4
// stages, the warp's lane 0 refilling a stage as soon as the warp has consumed it; no block-wide
// barrier exists until the final reduction.  Within a warp, lane = 10 u + t computes the 8 x 8
// tile t of the upper triangle of 32 x 32 tiles (10 tiles) for vector 3 it + u of the box
// (lanes 30, 31 idle), with paired FP32 FMAs (fma.rn.f32x2): 32 issue slots per 64 FMAs.
// ---------------------------------------------------------------------------------------
constexpr int G32_VPS = 48;     // vectors per TMA box (one stage)
constexpr int G32_STAGES = 4;   // stages per warp
constexpr int G32_WARPS = 8;
constexpr int G32_FLUSH = 4;    // stages (64 vectors per lane) between FP64 flushes
constexpr uint32_t G32_STAGE_BYTES = G32_VPS * 128;
constexpr size_t G32_RING = (size_t)G32_WARPS * G32_STAGES * G32_STAGE_BYTES;
constexpr size_t G32_SMEM = 1024 + G32_RING + (size_t)G32_WARPS * G32_STAGES * 8;
static_assert(G32_RING >= 256 * 65 * sizeof(double), "reduction area fits in the stage ring");

__device__ __forceinline__ float4 lds_f4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}
__device__ __forceinline__ void lds_u2(uint32_t addr, uint64_t& a, uint64_t& b) {
  asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"(addr));
}

__global__ void __launch_bounds__(256, 1)
    k_gram32x(const __grid_constant__ CUtensorMap tm, long long nvec, double* __restrict__ part, DevStatus* st) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t wbase = smem_u32(smem) + (uint32_t)(warp * G32_STAGES) * G32_STAGE_BYTES;
  const Bars bars{smem_u32(smem + G32_RING) + 8u * G32_STAGES * warp, G32_STAGES};
  if (lane == 0) {
    for (int s = 0; s < G32_STAGES; ++s) mbar_init(bars.full(s), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tm) : "memory");
  }
  __syncwarp();
  const long long nchunk = (nvec + G32_VPS - 1) / G32_VPS;
  const long long gw = (long long)blockIdx.x * G32_WARPS + warp;
  const long long GW = (long long)gridDim.x * G32_WARPS;
  const long long my = gw < nchunk ? (nchunk - 1 - gw) / GW + 1 : 0;  // boxes of this warp
  if (lane == 0) {
    for (int s = 0; s < G32_STAGES && s < my; ++s) {
      mbar_expect_tx(bars.full(s), G32_STAGE_BYTES);
      tma_load_2d(wbase + s * G32_STAGE_BYTES, &tm, bars.full(s), 0, (int)((gw + s * GW) * G32_VPS));
    }
  }
  const int t = lane % 10, u = lane / 10;
  const int p = t < 4 ? 0 : t < 7 ? 1 : t < 9 ? 2 : 3;
  const int q = t < 4 ? t : t < 7 ? t - 3 : t < 9 ? t - 5 : 3;
  uint64_t acc[8][4];  // (W[8p+i][8q+2j], W[8p+i][8q+2j+1])
  double accd[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0ull;
#pragma unroll
    for (int j = 0; j < 8; ++j) accd[i][j] = 0.0;
  }
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float lo, hi;
        f2_unpack(acc[i][j], lo, hi);
        accd[i][2 * j] += (double)lo;
        accd[i][2 * j + 1] += (double)hi;
        acc[i][j] = 0ull;
      }
  };
  long long k = 0;
  bool ok = true;
  for (; k < my; ++k) {
    const int s = (int)(k % G32_STAGES);
    ok = mbar_wait_limit(bars.full(s), (uint32_t)((k / G32_STAGES) & 1));
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) break;
    const uint32_t sb = wbase + (uint32_t)s * G32_STAGE_BYTES;
    if (u < 3) {
#pragma unroll 2
      for (int it = 0; it < G32_VPS / 3; ++it) {
        const int v = 3 * it + u;
        const uint32_t row = sb + (uint32_t)v * 128u;
        const int sw = v & 7;
        const float4 a0 = lds_f4(row + ((uint32_t)((2 * p) ^ sw) << 4));
        const float4 a1 = lds_f4(row + ((uint32_t)((2 * p + 1) ^ sw) << 4));
        uint64_t b[4];
        lds_u2(row + ((uint32_t)((2 * q) ^ sw) << 4), b[0], b[1]);
        lds_u2(row + ((uint32_t)((2 * q + 1) ^ sw) << 4), b[2], b[3]);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const uint64_t ad = f2_dup(a[i]);
#pragma unroll
          for (int j = 0; j < 4; ++j) ffma2(acc[i][j], ad, b[j]);
        }
      }
    }
    __syncwarp();
    if (lane == 0 && k + G32_STAGES < my) {
      // the warp's reads of this stage are done; order them before the async-proxy refill
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bars.full(s), G32_STAGE_BYTES);
      tma_load_2d(sb, &tm, bars.full(s), 0, (int)((gw + (k + G32_STAGES) * GW) * G32_VPS));
    }
    if ((k % G32_FLUSH) == G32_FLUSH - 1) flush();
  }
  flush();
  if (!ok) {
    if (lane == 0) {
      dev_fail(st, TT_ERR_TIMEOUT, 4);
      // every issued fill must land before the CTA leaves (fills issued: min(my, k + STAGES))
      drain_fills(bars, G32_STAGES, my < k + G32_STAGES ? my : k + G32_STAGES);
    }
    __syncwarp();
  }
  __syncthreads();  // every warp is done with its ring: reuse it for the block reduction
  double* red = reinterpret_cast<double*>(smem);
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) red[tid * 65 + i * 8 + j] = accd[i][j];
  __syncthreads();
  double* dst = part + (long long)blockIdx.x * 1024;
  for (int e = tid; e < 10 * 64; e += blockDim.x) {
    const int tt = e >> 6, ij = e & 63;
    double sum = 0.0;
    for (int w = 0; w < G32_WARPS; ++w)
      for (int uu = 0; uu < 3; ++uu) sum += red[(w * 32 + uu * 10 + tt) * 65 + ij];
    const int pp = tt < 4 ? 0 : tt < 7 ? 1 : tt < 9 ? 2 : 3;
    const int qq = tt < 4 ? tt : tt < 7 ? tt - 3 : tt < 9 ? tt - 5 : 3;
    dst[(8 * pp + (ij >> 3)) * 32 + 8 * qq + (ij & 7)] = sum;
  }
}

// W (M x M, column-major) = sum over blocks of the upper-tile partials (fixed order).
__global__ void k_gram32x_finish(const double* __restrict__ part, int nblk, int M, double* __restrict__ w) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * M; e += gridDim.x * blockDim.x) {
    const int i = e % M, j = e / M;
    const int r = i < j ? i : j, c = i < j ? j : i;
    double sum = 0.0;
    for (int b = 0; b < nblk; ++b) sum += part[(long long)b * 1024 + r * 32 + c];
    w[e] = sum;
  }
}

// Self-test of the bounded wait: one warp waits (with the pipeline limit and the abort-flag
// path of the tensor-core kernels) on an mbarrier that nothing ever arrives at, and reports
// TT_ERR_TIMEOUT through the status word when the limit runs out.  No copy or MMA is in flight,
// so the CTA can leave at once.
__global__ void k_wait_selftest(DevStatus* st) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (!mbar_wait(smem_u32(&bar), 0, &abort_flag)) dev_fail(st, TT_ERR_TIMEOUT, 99);
  }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;  // process-wide driver entry point
constexpr int kMaxTcDev = 64;
int g_tc_state[kMaxTcDev];  // per device: 0 unknown, 1 unavailable, 2 available

// Tensor-core engine availability of the current device (its compute capability decides).
bool init_tc() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int* state = (dev >= 0 && dev < kMaxTcDev) ? &g_tc_state[dev] : nullptr;
  if (state && *state) return *state == 2;
  bool ok = false;
  const char* dis = getenv("TTR_DISABLE_TC");
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (!(dis && dis[0] == '1') && major == 10) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn) {
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
      ok = true;
    } else {
      cudaGetLastError();
    }
  }
  if (state) *state = ok ? 2 : 1;
  return ok;
}

int make_map(CUtensorMap* map, const void* base, unsigned long long d0, unsigned long long d1,
             unsigned long long stride1_bytes, unsigned b0, unsigned b1, CUtensorMapSwizzle sw,
             CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32) {
  cuuint64_t dims[2] = {d0, d1};
  cuuint64_t strides[1] = {stride1_bytes};
  cuuint32_t box[2] = {b0, b1};
  cuuint32_t es[2] = {1, 1};
  CUresult r = g_encode(map, dt, 2, const_cast<void*>(base), dims, strides,
                        box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error(TT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) dims %llu x %llu box %u x %u", (int)r, d0, d1,
              b0, b1);
    return TT_ERR_CUDA;
  }
  return TT_OK;
}

// 3-D map over a column-major m x n FP32 matrix viewed as (32 rows of a block, column, block):
// strides m*4 bytes (column) and 128 bytes (block), box (32, bk, nblk).  One copy then fills
// nblk consecutive 32-row blocks of bk columns each, laid out block after block.
int make_map_blocks(CUtensorMap* map, const float* base, unsigned long long m, unsigned long long n,
                    unsigned bk, unsigned nblk, CUtensorMapSwizzle sw, CUtensorMapDataType dt) {
  cuuint64_t dims[3] = {32, n, m / 32};
  cuuint64_t strides[2] = {m * 4, 128};
  cuuint32_t box[3] = {32, bk, nblk};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(map, dt, 3, const_cast<float*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? TT_OK : TT_ERR_UNSUPPORTED;
}

template <typename K>
int set_smem(K kernel, size_t bytes) {
  return smem_optin(reinterpret_cast<const void*>(kernel), bytes);
}

constexpr size_t kSmemBudget = 200 * 1024;

// Round-to-nearest-even FP32 -> TF32 (10 stored mantissa bits) and the exact remainder.
__device__ __forceinline__ float tf32_rn(float x) {
  uint32_t u = __float_as_uint(x);
  if ((u & 0x7F800000u) != 0x7F800000u) {
    u += 0x0FFFu + ((u >> 13) & 1u);
    u &= 0xFFFFE000u;
  }
  return __uint_as_float(u);
}

__global__ void k_split_tf32(const float* __restrict__ q, long long m, int N, long long ldq,
                             float* __restrict__ hi, float* __restrict__ lo, long long ldo) {
  const long long total = m * (long long)N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx % m, c = idx / m;
    const float v = q[i + ldq * c];
    const float h = tf32_rn(v);
    hi[i + ldo * c] = h;
    lo[i + ldo * c] = v - h;
  }
}

template <int BN, bool SPLIT>
int run_project(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mb2, long long n,
                int N, int KB, float* out, long long ldo, int mode, int r0, int r1, DevStatus* st,
                cudaStream_t s) {
  constexpr uint32_t STAGE = 128 * 128 + (SPLIT ? 2 : 1) * BN * 128;
  // bond-permute staging of the 8 epilogue warps (that epilogue runs for BN <= 32 only)
  constexpr size_t STAGING = BN <= 32 ? 8 * 32 * (BN + 1) * sizeof(float) : 0;
  constexpr int STAGES = (int)std::min<size_t>(10, (kSmemBudget - STAGING) / STAGE);
  const size_t smem = (size_t)STAGES * STAGE + 1024 + 256 + STAGING;
  auto kern = k_project_tc<BN, STAGES, SPLIT>;
  if (set_smem(kern, smem) != TT_OK) return TT_ERR_CUDA;
  const long long ntiles = (n + 127) / 128;
  const int grid = (int)std::min<long long>(ntiles, (long long)dev_sms());
  kern<<<grid, 320, smem, s>>>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

template <int BN, int MT>
int run_sketch(const CUtensorMap& ma, const CUtensorMap& mb, long long m, long long n, int N,
               long long kchunk, int nsplit, int ngroups, double* part, DevStatus* st, cudaStream_t s,
               int a3d) {
  constexpr int BK = MT >= 8 ? 8 : MT == 4 ? 16 : 32;
  constexpr uint32_t STAGE = ((MT * 4) * BK * 128 + BN * BK * 4 + 1023) & ~1023u;
  constexpr int STAGES = (int)std::min<size_t>(8, kSmemBudget / STAGE);
  const size_t smem = (size_t)STAGES * STAGE + 1024 + 256;
  auto kern = k_sketch_tc<BN, MT, BK, STAGES>;
  if (set_smem(kern, smem) != TT_OK) return TT_ERR_CUDA;
  const int units = ngroups * nsplit;
  const int grid = std::min(units, dev_sms());
  kern<<<grid, 192, smem, s>>>(ma, mb, m, n, N, kchunk, nsplit, ngroups, part, st, a3d);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

int pad_bn(int N) { return N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : N <= 64 ? 64 : 128; }

int sketch_tc_plan(long long m, long long n, int N, int* MT, int* ngroups, int* nsplit, long long* kchunk) {
  const int BN = pad_bn(N);
  const int BNP = (BN + 15) / 16 * 16;
  int mt = (int)std::min<long long>(8, (m + 127) / 128);
  mt = mt >= 8 ? 8 : mt >= 4 ? 4 : mt >= 2 ? 2 : 1;
  while (mt > 1 && mt * BNP > 512) mt /= 2;
  const int bk = mt >= 8 ? 8 : mt == 4 ? 16 : 32;
  const int ng = (int)((m + mt * 128 - 1) / (mt * 128));
  const int sms = dev_sms();
  int ns = std::max(1, sms / ng);
  long long kc = (n + ns - 1) / ns;
  kc = std::max<long long>(kc, 4LL * bk);
  kc = (kc + bk - 1) / bk * bk;
  ns = (int)((n + kc - 1) / kc);
  *MT = mt;
  *ngroups = ng;
  *nsplit = ns;
  *kchunk = kc;
  return BN;
}


template <int NB>
int run_gram(const CUtensorMap& ma, long long ncols, int m, int grouped, long long kchunk, int nsplit,
             double* part, DevStatus* st, cudaStream_t s) {
  constexpr uint32_t STAGE = 4 * 32 * 128;
  constexpr int STAGES = 8;  // 128 KB ring + the m x (m+1) Gram accumulator
  const size_t smem = (size_t)STAGES * STAGE + 1024 + 256 + (size_t)m * (m + 1) * sizeof(float);
  auto kern = k_gram_tc<NB, STAGES>;
  {
    const size_t most = (size_t)STAGES * STAGE + 1024 + 256 + 128 * 129 * sizeof(float);
    if (set_smem(kern, most) != TT_OK) return TT_ERR_CUDA;
  }
  const int grid = std::min(nsplit, dev_sms());
  kern<<<grid, 192, smem, s>>>(ma, ncols, m, grouped, kchunk, nsplit, part, st);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

void gram_tc_plan(long long m, long long n, int* grouped, long long* ncols, int* nsplit,
                  long long* kchunk) {
  const bool g = (128 % m == 0) && ((n * m) % 128 == 0);
  *grouped = g ? 1 : 0;
  *ncols = g ? (n * m) / 128 : n;
  // Each unit's MMA accumulation runs in FP32 (TMEM); units of at most 2048 columns keep its
  // rounding small before the FP64 sum of the unit partials.
  const int sms = dev_sms();
  long long kc = (*ncols + sms - 1) / sms;
  kc = std::min<long long>(std::max<long long>(kc, 128), 2048);
  kc = (kc + 31) / 32 * 32;
  *kchunk = kc;
  *nsplit = (int)((*ncols + kc - 1) / kc);
}

}  // namespace

size_t gram_tc_ws_bytes(long long m, long long n) {
  if (!init_tc() || m > 128) return 0;
  int grouped, ns;
  long long nc, kc;
  gram_tc_plan(m, n, &grouped, &nc, &ns, &kc);
  return (size_t)ns * m * m * sizeof(double) + 4096;
}

// W (m x m, FP64) = A A^T with the tensor cores; A column-major m x n, m <= 128.
int launch_gram_tc(const float* a, long long m, long long n, double* w, Arena& ws, DevStatus* st,
                   cudaStream_t s) {
  if (!init_tc()) return TT_ERR_UNSUPPORTED;
  if (m < 1 || m > 128 || (m & 3) || (reinterpret_cast<uintptr_t>(a) & 15) || n > (1LL << 31) - 256)
    return TT_ERR_UNSUPPORTED;
  int grouped, ns;
  long long nc, kc;
  gram_tc_plan(m, n, &grouped, &nc, &ns, &kc);
  const size_t mk = ws.mark();
  double* part = ws.take<double>((size_t)ns * m * m);
  if (!part) {
    set_error(TT_ERR_NOMEM, "gram_tc workspace");
    return TT_ERR_NOMEM;
  }
  CUtensorMap ma;
  const unsigned long long rows = grouped ? 128ull : (unsigned long long)m;
  TT_TRY(make_map(&ma, a, rows, (unsigned long long)nc, rows * 4, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                  CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  const int NB = grouped ? 128 : (int)((m + 15) / 16 * 16);
  int rc;
  switch (NB) {
    case 16: rc = run_gram<16>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 32: rc = run_gram<32>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 48: rc = run_gram<48>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 64: rc = run_gram<64>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 80: rc = run_gram<80>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 96: rc = run_gram<96>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    case 112: rc = run_gram<112>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
    default: rc = run_gram<128>(ma, nc, (int)m, grouped, kc, ns, part, st, s); break;
  }
  if (rc != TT_OK) return rc;
  TT_TRY(launch_reduce_splits(part, m * m, ns, w, s));
  ws.reset(mk);
  return TT_OK;
}

bool tc_available() { return init_tc(); }

int set_wait_limit_ns(unsigned long long ns) {
  const unsigned long long v = ns ? ns : kWaitLimitNs;
  TT_CUDA(cudaMemcpyToSymbol(g_wait_limit_ns, &v, sizeof(v)));
  return TT_OK;
}

int launch_wait_selftest(DevStatus* st, cudaStream_t s) {
  k_wait_selftest<<<1, 32, 0, s>>>(st);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

size_t gram32x_ws_bytes() { return (size_t)dev_sms() * 1024 * sizeof(double) + 4096; }

// Exact Gram of nvec contiguous M-float vectors (M <= 32, M % 4 == 0, 16-byte aligned) on the
// CUDA cores; TT_ERR_UNSUPPORTED (nothing launched) when the shape or the device does not fit.
int launch_gram32x(const float* x, long long nvec, int M, double* w, Arena& ws, DevStatus* st, cudaStream_t s) {
  if (!init_tc()) return TT_ERR_UNSUPPORTED;
  if (M < 1 || M > 32 || (M & 3) || nvec < 1 || (reinterpret_cast<uintptr_t>(x) & 15) ||
      nvec > (1LL << 31) - 2 * G32_VPS)
    return TT_ERR_UNSUPPORTED;
  CUtensorMap map;
  {
    cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)nvec};
    cuuint64_t strides[1] = {(cuuint64_t)M * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)G32_VPS};
    cuuint32_t es[2] = {1, 1};
    const CUresult r = g_encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(x), dims, strides,
                                box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return TT_ERR_UNSUPPORTED;
  }
  const long long nchunk = (nvec + G32_VPS - 1) / G32_VPS;
  const int grid = (int)std::max<long long>(1, std::min<long long>(dev_sms(), ceil_div_ll(nchunk, G32_WARPS)));
  const size_t mk = ws.mark();
  double* part = ws.take<double>((size_t)grid * 1024);
  if (!part) {
    set_error(TT_ERR_NOMEM, "gram32x workspace");
    return TT_ERR_NOMEM;
  }
  TT_TRY(set_smem(k_gram32x, G32_SMEM));
  k_gram32x<<<grid, 256, G32_SMEM, s>>>(map, nvec, part, st);
  count_launch();
  TT_LAUNCH_CHECK();
  k_gram32x_finish<<<ceil_div(M * M, 256), 256, 0, s>>>(part, grid, M, w);
  count_launch();
  TT_LAUNCH_CHECK();
  ws.reset(mk);
  return TT_OK;
}


size_t sketch_tc_ws_bytes(long long m, long long n, int N) {
  if (!init_tc()) return 0;
  int mt, ng, ns;
  long long kc;
  sketch_tc_plan(m, n, N, &mt, &ng, &ns, &kc);
  return (size_t)ns * N * m * sizeof(double) + 4096;
}

int launch_project_tc(const float* a, long long m, long long n, const float* q, int N,
                      long long ldq, float* out, long long ldo, int mode, int r0, int r1,
                      Arena& ws, DevStatus* st, cudaStream_t s) {
  if (!init_tc()) return TT_ERR_UNSUPPORTED;
  if (N > 128 || (m & 3) || (reinterpret_cast<uintptr_t>(a) & 15) || n > (1LL << 31) - 256 ||
      m > (1LL << 31))
    return TT_ERR_UNSUPPORTED;
  const int BN = pad_bn(N);
  if (mode == OUT_PERM231 && BN > 32) return TT_ERR_UNSUPPORTED;
  // Q = Qhi + Qlo, Qhi exactly representable in TF32 (round to nearest), Qlo the FP32 remainder.
  const size_t mk = ws.mark();
  const long long ldh = (m + 3) & ~3LL;
  float* qhi = ws.take<float>((size_t)ldh * N);
  float* qlo = ws.take<float>((size_t)ldh * N);
  if (!qhi || !qlo) {
    set_error(TT_ERR_NOMEM, "project_tc workspace");
    return TT_ERR_NOMEM;
  }
  {
    const long long total = m * (long long)N;
    const int grid = (int)std::min<long long>((total + 255) / 256, 4LL * dev_sms());
    k_split_tf32<<<grid, 256, 0, s>>>(q, m, N, ldq, qhi, qlo, ldh);
    count_launch();
    TT_LAUNCH_CHECK();
  }
  CUtensorMap ma, mb, mb2;
  // A through the TFLOAT32 tensor-map type; the MMA then sees TMA-converted operands.
  TT_TRY(make_map(&ma, a, (unsigned long long)m, (unsigned long long)n, (unsigned long long)m * 4, 32, 128,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  TT_TRY(make_map(&mb, qhi, (unsigned long long)m, (unsigned long long)N, (unsigned long long)ldh * 4, 32,
                  (unsigned)BN, CU_TENSOR_MAP_SWIZZLE_128B));
  TT_TRY(make_map(&mb2, qlo, (unsigned long long)m, (unsigned long long)N, (unsigned long long)ldh * 4, 32,
                  (unsigned)BN, CU_TENSOR_MAP_SWIZZLE_128B));
  const int KB = (int)((m + 31) / 32);
  int rc;
  switch (BN) {
    case 16: rc = run_project<16, true>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st, s); break;
    case 32: rc = run_project<32, true>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st, s); break;
    case 48: rc = run_project<48, true>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st, s); break;
    case 64: rc = run_project<64, true>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st, s); break;
    default: rc = run_project<128, true>(ma, mb, mb2, n, N, KB, out, ldo, mode, r0, r1, st, s); break;
  }
  ws.reset(mk);  // the split copies are consumed by the launch above (stream-ordered)
  return rc;
}

int launch_sketch_tc(const float* a, long long m, long long n, const float* w, int N, long long wj,
                     long long wc, double* y, Arena& ws, DevStatus* st, cudaStream_t s) {
  if (!init_tc()) return TT_ERR_UNSUPPORTED;
  // W must be K-major (column-major n x N); the row-major power-iteration operand stays on the
  // plain-FP32 kernel.
  if (wj != 1 || N > 128 || (m & 31) || (wc & 3) || (reinterpret_cast<uintptr_t>(a) & 15) ||
      (reinterpret_cast<uintptr_t>(w) & 15) || n > (1LL << 31) - 256 || m > (1LL << 31))
    return TT_ERR_UNSUPPORTED;
  int MT, ng, ns;
  long long kc;
  const int BN = sketch_tc_plan(m, n, N, &MT, &ng, &ns, &kc);
  const int BK = MT >= 8 ? 8 : MT == 4 ? 16 : 32;
  const size_t mk = ws.mark();
  double* part = ws.take<double>((size_t)ns * N * m);
  if (!part) {
    set_error(TT_ERR_NOMEM, "sketch_tc workspace");
    return TT_ERR_NOMEM;
  }
  CUtensorMap ma, mb;
  // One 3-D copy per stage when the driver accepts the block view (MT*4 blocks of 32 rows),
  // otherwise one 2-D copy per 32-row block.
  int a3d = 0;
  if (!getenv("TTR_SKETCH_2D") &&
      make_map_blocks(&ma, a, (unsigned long long)m, (unsigned long long)n, (unsigned)BK, (unsigned)(MT * 4),
                      CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32) == TT_OK)
    a3d = 1;
  else
    TT_TRY(make_map(&ma, a, (unsigned long long)m, (unsigned long long)n, (unsigned long long)m * 4, 32,
                    (unsigned)BK, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  const CUtensorMapSwizzle bsw = BK == 8 ? CU_TENSOR_MAP_SWIZZLE_32B
                                 : BK == 16 ? CU_TENSOR_MAP_SWIZZLE_64B
                                            : CU_TENSOR_MAP_SWIZZLE_128B;
  TT_TRY(make_map(&mb, w, (unsigned long long)n, (unsigned long long)N, (unsigned long long)wc * 4,
                  (unsigned)BK, (unsigned)BN, bsw, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  int rc;
#define SK(BNV, MTV) rc = run_sketch<BNV, MTV>(ma, mb, m, n, N, kc, ns, ng, part, st, s, a3d)
#define SK_MT(BNV)                   \
  switch (MT) {                      \
    case 8: SK(BNV, 8); break;       \
    case 4: SK(BNV, 4); break;       \
    case 2: SK(BNV, 2); break;       \
    default: SK(BNV, 1); break;      \
  }
  switch (BN) {
    case 16: SK_MT(16); break;
    case 32: SK_MT(32); break;
    case 48: SK_MT(48); break;
    case 64: SK_MT(64); break;
    default:
      switch (MT) {
        case 4: SK(128, 4); break;
        case 2: SK(128, 2); break;
        default: SK(128, 1); break;
      }
      break;
  }
#undef SK_MT
#undef SK
  if (rc != TT_OK) return rc;
  const long long count = (long long)N * m;
  TT_TRY(launch_reduce_splits(part, count, ns, y, s));
  ws.reset(mk);
  return TT_OK;
}


// Sketch with the split-K partials in caller-provided scratch (`part`, `part_cap` doubles): the
// split count is lowered until the partials fit.  Allocates nothing.
int launch_sketch_tc_static(const float* a, long long m, long long n, const float* w, int N,
                            long long wj, long long wc, double* y, double* part, size_t part_cap,
                            DevStatus* st, cudaStream_t s) {
  if (!init_tc()) return TT_ERR_UNSUPPORTED;
  if (wj != 1 || N > 128 || (m & 31) || (wc & 3) || (reinterpret_cast<uintptr_t>(a) & 15) ||
      (reinterpret_cast<uintptr_t>(w) & 15) || n > (1LL << 31) - 256 || m > (1LL << 31))
    return TT_ERR_UNSUPPORTED;
  int MT, ng, ns;
  long long kc;
  const int BN = sketch_tc_plan(m, n, N, &MT, &ng, &ns, &kc);
  const int BK = MT >= 8 ? 8 : MT == 4 ? 16 : 32;
  const long long max_ns = (long long)(part_cap / ((size_t)N * (size_t)m));
  if (max_ns < 1) {
    set_error(TT_ERR_SHAPE, "sketch partials of %lld x %d doubles exceed the scratch of %zu doubles", m, N,
              part_cap);
    return TT_ERR_SHAPE;
  }
  if (ns > max_ns) {
    kc = (n + max_ns - 1) / max_ns;
    kc = (kc + BK - 1) / BK * BK;
    ns = (int)((n + kc - 1) / kc);
  }
  CUtensorMap ma, mb;
  // One 3-D copy per stage when the driver accepts the block view (MT*4 blocks of 32 rows),
  // otherwise one 2-D copy per 32-row block.
  int a3d = 0;
  if (!getenv("TTR_SKETCH_2D") &&
      make_map_blocks(&ma, a, (unsigned long long)m, (unsigned long long)n, (unsigned)BK, (unsigned)(MT * 4),
                      CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32) == TT_OK)
    a3d = 1;
  else
    TT_TRY(make_map(&ma, a, (unsigned long long)m, (unsigned long long)n, (unsigned long long)m * 4, 32,
                    (unsigned)BK, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  const CUtensorMapSwizzle bsw = BK == 8 ? CU_TENSOR_MAP_SWIZZLE_32B
                                 : BK == 16 ? CU_TENSOR_MAP_SWIZZLE_64B
                                            : CU_TENSOR_MAP_SWIZZLE_128B;
  TT_TRY(make_map(&mb, w, (unsigned long long)n, (unsigned long long)N, (unsigned long long)wc * 4,
                  (unsigned)BK, (unsigned)BN, bsw, CU_TENSOR_MAP_DATA_TYPE_TFLOAT32));
  int rc;
#define SK(BNV, MTV) rc = run_sketch<BNV, MTV>(ma, mb, m, n, N, kc, ns, ng, part, st, s, a3d)
#define SK_MT(BNV)                   \
  switch (MT) {                      \
    case 8: SK(BNV, 8); break;       \
    case 4: SK(BNV, 4); break;       \
    case 2: SK(BNV, 2); break;       \
    default: SK(BNV, 1); break;      \
  }
  switch (BN) {
    case 16: SK_MT(16); break;
    case 32: SK_MT(32); break;
    case 48: SK_MT(48); break;
    case 64: SK_MT(64); break;
    default:
      switch (MT) {
        case 4: SK(128, 4); break;
        case 2: SK(128, 2); break;
        default: SK(128, 1); break;
      }
      break;
  }
#undef SK_MT
#undef SK
  if (rc != TT_OK) return rc;
  return launch_reduce_splits(part, (long long)N * m, ns, y, s);
}

}  // namespace ttr
