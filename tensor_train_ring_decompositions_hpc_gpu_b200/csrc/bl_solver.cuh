// Brent-Luk parallel Jacobi eigen-solver for N <= 64, shared by the single-matrix solver and the
// batched kernel.
#pragma once
#include <math.h>

#include "jacobi_rot.cuh"

namespace ttr {

// Small-N variant (N <= 64): parallel cyclic Jacobi in the Brent-Luk layout.
// W is stored by physical position: the two indices of rotation pair k always sit at positions
// 2k and 2k+1, so a round is a block-local update W' = J^T W J (each 2 x 2 block of W from itself
// and the two rotations of its row and column pairs), written straight to the positions the
// indices take next round.  The round-robin tournament moves every index but index 0 by one slot
// per round, which in positions is a shear: even positions move down one pair, odd ones up one
// pair (mv below, with the two ends turning round).  W is kept in its upper triangle only (each
// entry stored once, at its upper position), which halves the scattered stores; a block row is
// read as one 16-byte load; W is symmetrised on input ((W + W^T) / 2).
// The warps split three ways each round, with one barrier per round:
//   - the W warps update the upper 2 x 2 blocks, one per thread;
//   - the V warps hold the eigenvectors in registers.  For N <= 32 one warp does it all: lane i
//     keeps row i of V by position (Np registers), applies the round's Np / 2 rotations and the
//     shear as a fixed register permutation (compiled per Np), so no eigenvector entry leaves its
//     thread.  It runs one round behind, with the FP64 rotations that the W threads of the
//     diagonal blocks publish (they renormalise them anyway), and applies the last round after
//     the loop.  Moving V by shuffles or through shared memory every round costs more than the
//     rotation itself (the shuffle / shared-memory path is the round's bottleneck once all of V
//     crosses it).  For 32 < N <= 64 V is split by components: lane k of a V warp keeps positions
//     2k and 2k+1 of up to kBlVRows components and passes results on with two shuffles (lane k's
//     new even entry comes from lane k+1, its odd entry from lane k-1);
//   - the last warp computes the next round's rotations meanwhile, from the current blocks and
//     rotations (jacobi_cs32: two reciprocal square roots, no division).  The rotations are
//     published as FP32 pairs; the W and V warps renormalise them to FP64 (rot_from_cs32), while
//     the rotation warp forms the next round's 2 x 2 blocks from the FP32 pairs as they are: the
//     renormalisation scales both entries of a pair by the same factor 1 + O(1e-7), so those
//     blocks come out with relative errors of that size only (the off-diagonal entry included),
//     which moves the next rotation's angle by as much as FP32 (c, s) rounding does, and keeps
//     the renormalisation off the chain.  That chain bounds the round, so for N <= 48 it gets a
//     scheduler of its own: warps w with w % 4 == 3 (one scheduler's share, as warps are spread over the
//     four schedulers by w % 4) do no work but the barrier, and the W and V warps use the others
//     (measured 126 vs 178 us for N = 32; at N = 64 the W and V warps need all four).
// Pairs with a_pq^2 <= 1e-24 |a_pp a_qq| or |a_pq| <= 1e-14 max|diag| are not rotated
// (jacobi_needed); the solve ends after the first sweep that leaves no pair to rotate.
// Eigenvalues are ordered by a parallel rank count.
// Slot of index i in round-robin round r (slot 0 fixed, slots 1..NR cycle), and its position.
__device__ __forceinline__ int bl_slot(int i, int r, int NR) {
  if (i == 0) return 0;
  int v = i - 1 - r % NR;
  if (v < 0) v += NR;
  return 1 + v;
}
__device__ __forceinline__ int bl_pos(int x, int Np) { return x < Np / 2 ? 2 * x : 2 * (Np - 1 - x) + 1; }
// Next-round position of the entry at position P (Np >= 4): the Brent-Luk shear.
__host__ __device__ constexpr int bl_move(int P, int Np) {
  if (P & 1) return P + 2 < Np ? P + 2 : Np - 2;  // odd positions up one pair; the top one turns down
  return P >= 4 ? P - 2 : (P == 2 ? 1 : 0);       // even positions down one pair; 2 turns up, 0 stays
}

constexpr int kBlVRows = 5;  // eigenvector components per V warp (32 < N <= 64)

// One round of the row-resident V (N <= 32): v holds row i of V by position; rotate the NP / 2
// pairs with the FP64 rotations cs and move every result to its next-round position, in place.
// Pair k's results go to positions 2k - 2 (pair k - 1's even slot, or 0 / 1 for k = 0 / 1) and
// 2k + 3 (pair k + 1's odd slot, or NP - 2 for the last pair), so in increasing k every
// destination but the next pair's odd slot has been read already; that one old value is carried.
// The rotations are read 8 pairs at a time (a warp barrier between the groups keeps the compiler
// from loading all of them ahead, which would hold 4 NP more registers).
template <int NP, int VN>
__device__ __forceinline__ void bl_vrow_round(double (&v)[VN], const double2* __restrict__ cs) {
  if (NP == 2) {
    const double2 r = cs[0];
    const double a = v[0], b = v[1];
    v[0] = a * r.x - b * r.y;
    v[1] = a * r.y + b * r.x;
    return;
  }
  double ob = v[1];  // the old odd entry of the pair being rotated
#pragma unroll
  for (int k = 0; k < NP / 2; ++k) {
    if (k > 0 && k % 8 == 0) __syncwarp();
    const double2 r = cs[k];
    const double a = v[2 * k], b = ob;
    if (k + 1 < NP / 2) ob = v[2 * k + 3];
    v[bl_move(2 * k, NP)] = a * r.x - b * r.y;
    v[bl_move(2 * k + 1, NP)] = a * r.y + b * r.x;
  }
}
template <int VN>
__device__ __forceinline__ void bl_vrow_apply(int Np, double (&v)[VN], const double2* __restrict__ cs) {
  switch (Np) {
#define BL_VR(NP)                                  \
  case NP:                                         \
    if constexpr (NP <= VN) bl_vrow_round<NP, VN>(v, cs); \
    break;
    BL_VR(2) BL_VR(4) BL_VR(6) BL_VR(8) BL_VR(10) BL_VR(12) BL_VR(14) BL_VR(16)
    BL_VR(18) BL_VR(20) BL_VR(22) BL_VR(24) BL_VR(26) BL_VR(28) BL_VR(30) BL_VR(32)
    BL_VR(34) BL_VR(36) BL_VR(38) BL_VR(40) BL_VR(42) BL_VR(44) BL_VR(46) BL_VR(48)
#undef BL_VR
    default:
      break;
  }
}

// Launch shape of the solver: the block's warp count (the last one the rotation warp) and whether
// the rotation warp has a scheduler of its own (warps w % 4 == 3 idle), which needs the W warps
// (one block per thread) and the V warps to fit on three schedulers' 24 warp slots (N <= 48);
// larger N use every warp.  rowv: V row-resident (a row of V per lane, N <= 46), in at most 12
// warps (the registers of a row of V), so N = 45, 46 give up the rotation warp's scheduler.
__host__ __device__ inline void bl_shape(int N, bool rowv, int* iso, int* warps) {
  const int Np = N + (N & 1), H = Np / 2, NWB = H * (H + 1) / 2;
  const int nv = rowv ? (N + 31) / 32 : (N + kBlVRows - 1) / kBlVRows;
  const int wu = (NWB + 31) / 32;
  *iso = (wu + nv <= 24 && !(rowv && 4 * ((wu + nv + 2) / 3) > 12)) ? 1 : 0;
  *warps = *iso ? 4 * ((wu + nv + 2) / 3) : wu + nv + 1;
}

// The solve by the whole block (blockDim.x / 32 warps, a multiple of 4 and at least bl_shape's
// count): W (N x N, symmetric, any layout) -> evals (descending), evecs (N x N column-major);
// `wbuf` holds 2 (N + N % 2)^2 doubles of shared memory.  Returns the sweeps run, or
// max_sweeps + 1 when the last sweep still rotated.  Ends with a block barrier.
// VN: 32 or 48 keeps V row-resident and serves N <= min(VN, 46); 0 splits V by components
// (N <= 64).
template <int VN>
__device__ __forceinline__ int bl_solve(const double* __restrict__ w_in, int N, double* __restrict__ evals,
                                        double* __restrict__ evecs, int max_sweeps, double* wbuf) {
  static_assert(VN == 0 || VN == 32 || VN == 48, "bl_solve: VN is 0, 32 or 48");
  constexpr bool vrow = VN > 0;                      // V rows resident, one per lane of one warp
  const int PW = (int)(blockDim.x >> 5) - 1;  // the last warp computes the next round's rotations
  const int Np = N + (N & 1);
  const int NR = Np - 1;
  const int H = Np / 2;
  const int NN = Np * Np;
  double* Wb0 = wbuf;
  double* Wb1 = Wb0 + NN;
  __shared__ float2 pcs[2][32];   // FP32 (c, s) of each pair, current and next round
  __shared__ double2 pcd[2][32];  // the same renormalised to FP64, for the row-resident V
  __shared__ int imv[64];
  __shared__ double dg[64];
  __shared__ int rk[64], pidx[64];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int iso, nwarps;
  bl_shape(N, vrow, &iso, &nwarps);
  const int NWB = H * (H + 1) / 2;                   // upper blocks (a <= b), one per W thread
  const int WU = (NWB + 31) / 32;                    // W warps
  const int NVW = vrow ? (N + 31) / 32 : (N + kBlVRows - 1) / kBlVRows;  // V warps
  const int vrows = (N + NVW - 1) / NVW;             // components per V warp (<= kBlVRows)
  // role index among the working warps (with iso, those with w % 4 != 3); -1 for the idle ones
  // and the rotation warp
  const int ai = (warp == PW || (iso && (warp & 3) == 3)) ? -1 : iso ? (warp >> 2) * 3 + (warp & 3) : warp;
  const bool ww = ai >= 0 && ai < WU;                // W warp
  const bool vw = ai >= WU && ai < WU + NVW;         // V warp
  for (int P = tid; P < Np; P += blockDim.x) imv[Np >= 4 ? bl_move(P, Np) : P] = P;
  for (int idx = tid; idx < NN; idx += blockDim.x) {
    const int i = idx / Np, j = idx - (idx / Np) * Np;
    const int Pi = bl_pos(i, Np), Pj = bl_pos(j, Np);  // round 0: index i sits in slot i
    double x = 0.0;
    if (i < N && j < N) x = 0.5 * (w_in[i + (long long)N * j] + w_in[j + (long long)N * i]);
    Wb0[Pi * Np + Pj] = x;
  }
  double dm = 0.0;
  for (int i = 0; i < N; ++i) dm = fmax(dm, fabs(w_in[i + (long long)N * i]));
  const double inv_s = dm > 0.0 ? 1.0 / dm : 1.0;
  __syncthreads();
  // Rotations of round 0.
  if (warp == PW && lane < H) {
    const int k = lane;
    float2 cs = make_float2(1.0f, 0.0f);
    const int i0 = k, i1 = Np - 1 - k;  // indices in slots k and Np-1-k at round 0
    if (i0 < N && i1 < N)
      cs = jacobi_cs32(Wb0[(2 * k) * Np + 2 * k], Wb0[(2 * k + 1) * Np + 2 * k + 1], Wb0[(2 * k) * Np + 2 * k + 1],
                       inv_s);
    pcs[0][k] = cs;
  }
  __syncthreads();
  int R = 0;
  int sweep = 0;
  bool converged = false;
  // The round loop.  Each role runs it with its own body, so that one role's registers (the
  // row-resident V above all) are not live in another's code; every role takes the same barriers
  // in the same order.  A sweep ends with the convergence test: stop when no pair of the updated
  // matrix would be rotated (the following sweep would change nothing), which saves that quiet
  // sweep.
  auto rounds = [&](auto&& body) {
    for (; sweep < max_sweeps; ++sweep) {
      bool stop = false;
      for (int rnd = 0; rnd < NR; ++rnd, ++R) {
        body(rnd);
        __syncthreads();
        if (rnd + 1 == NR) {
          const double* Wn = (R & 1) ? Wb0 : Wb1;  // written this round
          int need = 0;
          for (int idx = tid; idx < NN; idx += blockDim.x) {
            const int P = idx / Np, Q = idx - (idx / Np) * Np;
            if (P < Q && jacobi_needed(Wn[P * Np + P], Wn[Q * Np + Q], Wn[P * Np + Q], inv_s)) need = 1;
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
  };
  const int vi0 = vw ? (ai - WU) * (vrow ? 32 : vrows) : 0;
  double v[vrow ? VN : 2 * kBlVRows];
  if (ww) {
    // W thread: upper block (a, b) of W, a <= b (a = -1 for none)
    int a = -1, b = 0;
    if (ai * 32 + lane < NWB) {
      int rem = ai * 32 + lane;
      a = 0;
      while (rem >= H - a) {
        rem -= H - a;
        ++a;
      }
      b = a + rem;
    }
    // next-round positions of the block's rows and columns
    const int r0 = Np >= 4 ? bl_move(2 * a, Np) : 0, r1 = Np >= 4 ? bl_move(2 * a + 1, Np) : 1;
    const int q0 = Np >= 4 ? bl_move(2 * b, Np) : 0, q1 = Np >= 4 ? bl_move(2 * b + 1, Np) : 1;
    rounds([&](int) {
      if (a < 0) return;
      const int cb = R & 1;
      const double* W = cb ? Wb1 : Wb0;
      double* Wn = cb ? Wb0 : Wb1;
      const float2* cs_ = pcs[cb];
      double ca, sa, cbv, sb;
      rot_from_cs32(cs_[a], ca, sa);
      rot_from_cs32(cs_[b], cbv, sb);
      if (vrow && a == b) pcd[cb][a] = make_double2(ca, sa);  // for V, next round
      // Only the upper triangle (row <= column) of W is kept.  Block (a, b), a < b, lies
      // wholly above the diagonal; a diagonal block's lower entry is its upper one.
      const double2 r0v = *reinterpret_cast<const double2*>(&W[(2 * a) * Np + 2 * b]);
      const double2 r1v = *reinterpret_cast<const double2*>(&W[(2 * a + 1) * Np + 2 * b]);
      const double w00 = r0v.x, w01 = r0v.y, w11 = r1v.y;
      const double w10 = (a == b) ? w01 : r1v.x;
      // X = J_a^T B: rows (c, -s), (s, c)
      const double x00 = ca * w00 - sa * w10, x01 = ca * w01 - sa * w11;
      const double x10 = sa * w00 + ca * w10, x11 = sa * w01 + ca * w11;
      // X J_b: columns (c, -s)^T, (s, c)^T
      const double y00 = x00 * cbv - x01 * sb, y01 = x00 * sb + x01 * cbv;
      const double y10 = x10 * cbv - x11 * sb, y11 = x10 * sb + x11 * cbv;
      // each entry to its upper position (a diagonal block's two off-diagonal entries are the
      // same entry)
      Wn[min(r0, q0) * Np + max(r0, q0)] = y00;
      Wn[min(r0, q1) * Np + max(r0, q1)] = y01;
      if (a != b) Wn[min(r1, q0) * Np + max(r1, q0)] = y10;
      Wn[min(r1, q1) * Np + max(r1, q1)] = y11;
    });
  } else if (vw) {
    // V, identity at the round-0 positions.  Row-resident: lane l of V warp j holds row
    // i = 32 j + l = vi0 + l, entry P in v[P].  Otherwise components vi0 .. vi0 + vrows - 1, entry
    // u of positions 2 lane and 2 lane + 1 in v[u] and v[kBlVRows + u].
    if constexpr (vrow) {
      const int Pi = vi0 + lane < N ? bl_pos(vi0 + lane, Np) : -1;
#pragma unroll
      for (int P = 0; P < VN; ++P) v[P] = (P == Pi) ? 1.0 : 0.0;
      rounds([&](int) {
        if (R > 0) bl_vrow_apply<VN>(Np, v, pcd[(R & 1) ^ 1]);  // the previous round's rotations
      });
      if (R > 0) bl_vrow_apply<VN>(Np, v, pcd[(R - 1) & 1]);  // and the last round's
    } else {
#pragma unroll
      for (int u = 0; u < kBlVRows; ++u) {
        const int i = vi0 + u;
        const int P = (u < vrows && i < N) ? bl_pos(i, Np) : -1;
        v[u] = (P == 2 * lane) ? 1.0 : 0.0;
        v[kBlVRows + u] = (P == 2 * lane + 1) ? 1.0 : 0.0;
      }
      rounds([&](int) {
        const float2* cs_ = pcs[R & 1];
        double c = 1.0, sn = 0.0;
        if (lane < H) rot_from_cs32(cs_[lane], c, sn);
#pragma unroll
        for (int u = 0; u < kBlVRows; ++u) {
          if (u >= vrows) break;  // uniform across the warp
          const double n0 = v[u] * c - v[kBlVRows + u] * sn;
          const double n1 = v[u] * sn + v[kBlVRows + u] * c;
          const double dn = __shfl_down_sync(0xffffffffu, n0, 1);  // lane k+1's even entry
          const double up = __shfl_up_sync(0xffffffffu, n1, 1);    // lane k-1's odd entry
          v[u] = lane == 0 ? n0 : (lane == H - 1 ? n1 : dn);
          v[kBlVRows + u] = lane == 0 ? dn : up;
        }
      });
    }
  } else if (warp == PW) {
    // Rotation of pair `lane` in the next round.  Its two indices sit at the current positions
    // P = imv[2 lane], Q = imv[2 lane + 1]; the three entries of J^T W J it needs come from the
    // 2 x 2 blocks (P/2, P/2), (Q/2, Q/2), (P/2, Q/2) and the rotations of pairs P/2 and Q/2 (row
    // x of J_a^T equals column x of J_a: (c, -s) or (s, c)).
    const int eP = lane < H ? imv[2 * lane] : 0, eQ = lane < H ? imv[2 * lane + 1] : 0;
    const int aP = eP >> 1, xP = eP & 1, aQ = eQ >> 1, xQ = eQ & 1;
    const int P0 = 2 * aP, Q0 = 2 * aQ;
    rounds([&](int rnd) {
      if (lane >= H) return;
      const int cb = R & 1;
      const double* W = cb ? Wb1 : Wb0;
      const float2* cs_ = pcs[cb];
      const int rn = (rnd + 1 == NR) ? 0 : rnd + 1;
      bool live = true;
      if (Np != N) {  // the padding index N = Np - 1 never rotates
        const int xs = bl_slot(Np - 1, rn, NR);
        live = (xs != lane) && (xs != Np - 1 - lane);
      }
      float2 cs = make_float2(1.0f, 0.0f);
      if (live) {
        const float2 fP = cs_[aP], fQ = cs_[aQ];  // FP32 pairs, not renormalised (see above)
        const double cP = fP.x, sP = fP.y, cQ = fQ.x, sQ = fQ.y;
        const double tP0 = xP ? sP : cP, tP1 = xP ? cP : -sP;
        const double tQ0 = xQ ? sQ : cQ, tQ1 = xQ ? cQ : -sQ;
        // entries through the upper triangle (W is kept there only); the address is selected
        // arithmetically, so the lanes do not diverge
        auto wu = [&](int r, int c2) { return W[min(r, c2) * Np + max(r, c2)]; };
        const double p0 = tP0 * wu(P0, P0) + tP1 * wu(P0, P0 + 1);
        const double p1 = tP0 * wu(P0, P0 + 1) + tP1 * wu(P0 + 1, P0 + 1);
        const double q0 = tQ0 * wu(Q0, Q0) + tQ1 * wu(Q0, Q0 + 1);
        const double q1 = tQ0 * wu(Q0, Q0 + 1) + tQ1 * wu(Q0 + 1, Q0 + 1);
        const double m0 = tP0 * wu(P0, Q0) + tP1 * wu(P0 + 1, Q0);
        const double m1 = tP0 * wu(P0, Q0 + 1) + tP1 * wu(P0 + 1, Q0 + 1);
        const double app = p0 * tP0 + p1 * tP1;
        const double aqq = q0 * tQ0 + q1 * tQ1;
        const double apq = m0 * tQ0 + m1 * tQ1;
        cs = jacobi_cs32(app, aqq, apq, inv_s);
      }
      pcs[cb ^ 1][lane] = cs;
    });
  } else {
    rounds([&](int) {});
  }
  // After R rounds the current buffer is (R & 1); index i sits in slot bl_slot(i, R, NR).
  const double* Wf = (R & 1) ? Wb1 : Wb0;
  if (tid < Np) pidx[tid] = -1;
  __syncthreads();
  if (tid < N) {
    const int P = bl_pos(bl_slot(tid, R, NR), Np);
    dg[tid] = Wf[P * Np + P];
    pidx[P] = tid;
  }
  __syncthreads();
  if (tid < N) {
    const int a = tid;
    double la = dg[a];
    if (la != la) la = -INFINITY;
    int rank = 0;
    for (int b = 0; b < N; ++b) {
      double lb = dg[b];
      if (lb != lb) lb = -INFINITY;
      rank += (lb > la || (lb == la && b < a)) ? 1 : 0;
    }
    rk[a] = rank;
    evals[rank] = dg[a];
  }
  __syncthreads();
  if constexpr (vrow) {
    if (vw && vi0 + lane < N) {
#pragma unroll
      for (int P = 0; P < VN; ++P) {
        const int a = P < Np ? pidx[P] : -1;  // index at position P
        if (a >= 0) evecs[vi0 + lane + (long long)N * rk[a]] = v[P];
      }
    }
  } else if (vw && lane < H) {
    const int a0 = pidx[2 * lane], a1 = pidx[2 * lane + 1];  // indices at this lane's positions
#pragma unroll
    for (int u = 0; u < kBlVRows; ++u) {
      const int i = vi0 + u;
      if (u >= vrows || i >= N) break;
      if (a0 >= 0) evecs[i + (long long)N * rk[a0]] = v[u];
      if (a1 >= 0) evecs[i + (long long)N * rk[a1]] = v[kBlVRows + u];
    }
  }
  __syncthreads();
  return converged ? sweep : max_sweeps + 1;
}

}  // namespace ttr
