// The learned EDrSVD parameter predictor: a 8 -> 64 -> 64 -> 3 ReLU network that maps cheap
// Gaussian-probe statistics of an unfolding to (truncation rank, oversampling, power
// iterations), with its own inference, gradient and training kernels.
//
// Parameters (FP32, packed): W1 (64 x 8, row-major), b1 (64), W2 (64 x 64), b2 (64),
// W3 (3 x 64), b3 (3).  Loss: mean over the batch of the summed squared error of the outputs;
// optimiser: bias-corrected Adam.
//
// Training runs in ONE persistent CTA of 512 threads for all steps: 8 groups of 64 threads each
// take every 8th sample of a minibatch, thread j of a group owning hidden unit j in both layers
// (forward: one row of W1 and W2; backward: the same rows of the gradients, accumulated in
// registers).  After a minibatch the 8 groups' partial gradients meet in shared memory, are summed
// in a fixed order and the Adam update is applied in place, so a run is bitwise reproducible.
// The network is tiny (4931 parameters): one CTA keeps it, its gradients and the partials in
// shared memory, and a training run of thousands of steps is a single launch.
//
// The reference has no learned component: its EDrSVD takes rank, oversampling and power count
// as fixed arguments (ttdec_gpu_float_rsvd_lu_half.cu:797-798, ttdec_gpu_float_edrsvd.cu:347-348).
#include <math.h>

#include "kernels.cuh"
#include "philox.cuh"

namespace ttr {
namespace {

constexpr int NI = TT_MLP_INPUTS, NH = 64, NO = TT_MLP_OUTPUTS;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NH * NI;
constexpr int OFF_W2 = OFF_B1 + NH;
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;
constexpr int OFF_B3 = OFF_W3 + NO * NH;
constexpr int NPARAM = OFF_B3 + NO;
static_assert(NPARAM == 4931, "parameter count");
constexpr int GROUPS = 8;
constexpr int TT_THREADS = GROUPS * NH;  // 512
constexpr int W2S = NH + 1;              // padded row stride of W2 in shared memory

// Shared memory of the training kernel (floats).
constexpr int SM_W2 = NH * W2S;
constexpr int SM_W3 = NO * NH;
constexpr int SM_B3 = 4;
constexpr int SM_H1 = GROUPS * NH;
constexpr int SM_D2 = GROUPS * NH;
constexpr int SM_RED = GROUPS * 2 * 4;
constexpr int SM_LOSS = GROUPS;
constexpr int SM_PART = GROUPS * NPARAM;
constexpr size_t TRAIN_SMEM =
    sizeof(float) * (size_t)(SM_W2 + SM_W3 + SM_B3 + SM_H1 + SM_D2 + SM_RED + SM_LOSS + SM_PART);

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(NH) : "memory");
}

// Where the partial gradient of parameter q sits in a group's partial block.  The weight
// matrices are stored transposed (input index major) so that the 64 threads of a group, each
// holding one row, write consecutive addresses.
__device__ __forceinline__ int part_slot(int q) {
  if (q < OFF_B1) {  // W1[j][i] at i*64 + j
    const int j = q / NI, i = q - j * NI;
    return OFF_W1 + i * NH + j;
  }
  if (q >= OFF_W2 && q < OFF_B2) {  // W2[j][i] at i*64 + j
    const int r = q - OFF_W2, j = r / NH, i = r - j * NH;
    return OFF_W2 + i * NH + j;
  }
  return q;  // biases, W3 (o*64 + j is already unit-major)
}

// mode 0: train `steps` Adam steps on minibatches of `batch` samples drawn from [0, n)
//         (Philox, with replacement);  mode 1: gradient of the loss over samples 0..batch-1
//         written to grad_out (no update).
__global__ void __launch_bounds__(TT_THREADS, 1)
    k_mlp_train(float* __restrict__ params, float* __restrict__ adam_m, float* __restrict__ adam_v,
                const float* __restrict__ x, const float* __restrict__ t, int n, int steps, int batch, float lr,
                int step0, unsigned long long seed, float* __restrict__ loss_trace, float* __restrict__ grad_out,
                int mode) {
  extern __shared__ __align__(16) float smf[];
  float* w2s = smf;
  float* w3s = w2s + SM_W2;
  float* b3s = w3s + SM_W3;
  float* h1s = b3s + SM_B3;
  float* d2s = h1s + SM_H1;
  float* red = d2s + SM_D2;
  float* lss = red + SM_RED;
  float* part = lss + SM_LOSS;

  const int tid = threadIdx.x;
  const int g = tid / NH, j = tid % NH, warp_in_group = j / 32, lane = tid & 31;
  float* h1g = h1s + g * NH;
  float* d2g = d2s + g * NH;
  float* redg = red + g * 8;
  float* partg = part + (size_t)g * NPARAM;
  const float inv_b = 1.0f / (float)batch;

  for (int step = 0; step < steps; ++step) {
    // weights of this step (after the previous update)
    float w1[NI], w3c[NO];
#pragma unroll
    for (int i = 0; i < NI; ++i) w1[i] = params[OFF_W1 + j * NI + i];
    const float b1 = params[OFF_B1 + j], b2 = params[OFF_B2 + j];
#pragma unroll
    for (int o = 0; o < NO; ++o) w3c[o] = params[OFF_W3 + o * NH + j];
    for (int q = tid; q < NH * NH; q += TT_THREADS) {
      const int r = q / NH, c = q - r * NH;
      w2s[r * W2S + c] = params[OFF_W2 + q];
    }
    if (tid < NO * NH) w3s[tid] = params[OFF_W3 + tid];
    if (tid < NO) b3s[tid] = params[OFF_B3 + tid];
    __syncthreads();

    float gw1[NI], gw2[NH], gw3[NO], gb1 = 0.f, gb2 = 0.f, gb3[NO], lacc = 0.f;
#pragma unroll
    for (int i = 0; i < NI; ++i) gw1[i] = 0.f;
#pragma unroll
    for (int i = 0; i < NH; ++i) gw2[i] = 0.f;
#pragma unroll
    for (int o = 0; o < NO; ++o) gw3[o] = gb3[o] = 0.f;

    for (int b = g; b < batch; b += GROUPS) {
      int idx;
      if (mode == 1) {
        idx = b;
      } else {
        const uint4 r = philox4x32_10(make_uint4((unsigned)(step0 + step), (unsigned)b, 0x4d4c50u, 0u),
                                      make_uint2((unsigned)(seed & 0xFFFFFFFFull), (unsigned)(seed >> 32)));
        idx = (int)(r.x % (unsigned)n);
      }
      float xi[NI];
#pragma unroll
      for (int i = 0; i < NI; ++i) xi[i] = x[(size_t)idx * NI + i];
      float z1 = b1;
#pragma unroll
      for (int i = 0; i < NI; ++i) z1 = fmaf(w1[i], xi[i], z1);
      const float h1 = fmaxf(z1, 0.f);
      h1g[j] = h1;
      group_sync(g);
      float z2 = b2;
#pragma unroll 16
      for (int i = 0; i < NH; ++i) z2 = fmaf(w2s[j * W2S + i], h1g[i], z2);
      const float h2 = fmaxf(z2, 0.f);
      float py[NO];
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        float v = w3c[o] * h2;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        py[o] = v;
      }
      if (lane == 0) {
#pragma unroll
        for (int o = 0; o < NO; ++o) redg[warp_in_group * 4 + o] = py[o];
      }
      group_sync(g);
      float dy[NO];
      float sq = 0.f;
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        const float y = b3s[o] + redg[o] + redg[4 + o];
        const float r = y - t[(size_t)idx * NO + o];
        sq = fmaf(r, r, sq);
        dy[o] = 2.f * r * inv_b;
        gw3[o] = fmaf(dy[o], h2, gw3[o]);
        gb3[o] += dy[o];
      }
      lacc += sq;
      float dh2 = 0.f;
#pragma unroll
      for (int o = 0; o < NO; ++o) dh2 = fmaf(w3c[o], dy[o], dh2);
      dh2 = z2 > 0.f ? dh2 : 0.f;
      d2g[j] = dh2;
      group_sync(g);
      float dh1 = 0.f;
#pragma unroll 16
      for (int i = 0; i < NH; ++i) dh1 = fmaf(w2s[i * W2S + j], d2g[i], dh1);
      dh1 = z1 > 0.f ? dh1 : 0.f;
#pragma unroll
      for (int i = 0; i < NH; ++i) gw2[i] = fmaf(dh2, h1g[i], gw2[i]);
      gb2 += dh2;
#pragma unroll
      for (int i = 0; i < NI; ++i) gw1[i] = fmaf(dh1, xi[i], gw1[i]);
      gb1 += dh1;
      group_sync(g);  // h1g, d2g and redg are rewritten by the next sample
    }
    // this group's partial gradients (weights transposed, see part_slot)
#pragma unroll
    for (int i = 0; i < NI; ++i) partg[OFF_W1 + i * NH + j] = gw1[i];
    partg[OFF_B1 + j] = gb1;
#pragma unroll
    for (int i = 0; i < NH; ++i) partg[OFF_W2 + i * NH + j] = gw2[i];
    partg[OFF_B2 + j] = gb2;
#pragma unroll
    for (int o = 0; o < NO; ++o) partg[OFF_W3 + o * NH + j] = gw3[o];
    if (j == 0) {
#pragma unroll
      for (int o = 0; o < NO; ++o) partg[OFF_B3 + o] = gb3[o];
      lss[g] = lacc;
    }
    __syncthreads();
    if (tid == 0 && loss_trace) {
      float l = 0.f;
      for (int q = 0; q < GROUPS; ++q) l += lss[q];
      loss_trace[step] = l * inv_b;
    }
    // fixed-order sum over the groups, then Adam (or the raw gradient in mode 1)
    const int tstep = step0 + step + 1;
    const double bc1 = 1.0 - pow(0.9, (double)tstep), bc2 = 1.0 - pow(0.999, (double)tstep);
    const float a_t = (float)(lr * sqrt(bc2) / bc1);
    for (int q = tid; q < NPARAM; q += TT_THREADS) {
      const int slot = part_slot(q);
      float gs = 0.f;
#pragma unroll
      for (int p = 0; p < GROUPS; ++p) gs += part[(size_t)p * NPARAM + slot];
      if (mode == 1) {
        grad_out[q] = gs;
      } else {
        const float m = 0.9f * adam_m[q] + 0.1f * gs;
        const float v = 0.999f * adam_v[q] + 0.001f * gs * gs;
        adam_m[q] = m;
        adam_v[q] = v;
        // bias-corrected step: lr * mhat / (sqrt(vhat) + eps), with mhat = m / bc1, vhat = v / bc2
        params[q] -= a_t * m / (sqrtf(v) + 1e-8f * sqrtf((float)bc2));
      }
    }
    __syncthreads();
  }
}

// Inference: one thread per sample, parameters in shared memory (read as broadcasts).
__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ x,
                                                     int n, float* __restrict__ y) {
  __shared__ float p[NPARAM];
  for (int q = threadIdx.x; q < NPARAM; q += blockDim.x) p[q] = params[q];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float xi[NI], h1[NH];
#pragma unroll
  for (int i = 0; i < NI; ++i) xi[i] = x[(size_t)s * NI + i];
#pragma unroll
  for (int jj = 0; jj < NH; ++jj) {
    float z = p[OFF_B1 + jj];
#pragma unroll
    for (int i = 0; i < NI; ++i) z = fmaf(p[OFF_W1 + jj * NI + i], xi[i], z);
    h1[jj] = fmaxf(z, 0.f);
  }
  float out[NO];
#pragma unroll
  for (int o = 0; o < NO; ++o) out[o] = p[OFF_B3 + o];
  for (int jj = 0; jj < NH; ++jj) {
    float z = p[OFF_B2 + jj];
#pragma unroll
    for (int i = 0; i < NH; ++i) z = fmaf(p[OFF_W2 + jj * NH + i], h1[i], z);
    const float h2 = fmaxf(z, 0.f);
#pragma unroll
    for (int o = 0; o < NO; ++o) out[o] = fmaf(p[OFF_W3 + o * NH + jj], h2, out[o]);
  }
#pragma unroll
  for (int o = 0; o < NO; ++o) y[(size_t)s * NO + o] = out[o];
}

// Probe features of an unfolding from the descending eigenvalues mu of Y^T Y (Y = A Omega,
// TT_PROBE_COLS Gaussian columns).  E[mu] follows the leading squared singular values and
// E[sum mu] = TT_PROBE_COLS ||A||_F^2, so the ratios describe the spectrum's decay and the
// share of the energy the leading directions hold.
__global__ void k_probe_features(const double* __restrict__ mu, double energy, double tol, long long m, long long n,
                                 float* __restrict__ out) {
  if (threadIdx.x != 0) return;
  const double mu1 = fmax(mu[0], 1e-300);
  const int idx[5] = {1, 3, 7, 11, 15};
  const double k = (double)(m < n ? m : n);
  out[0] = (float)(log2(k) / 10.0);
#pragma unroll
  for (int q = 0; q < 5; ++q) out[1 + q] = (float)(log10(fmax(mu[idx[q]], 1e-30 * mu1) / mu1) / 4.0);
  out[6] = (float)(log10(fmax((double)TT_PROBE_COLS * energy / mu1, 1e-30)) / 4.0);
  out[7] = (float)(log10(fmax(tol, 1e-30)) / 4.0);
}

int train_attr() { return smem_optin_k(k_mlp_train, TRAIN_SMEM); }

}  // namespace

int launch_probe_features(const double* mu, double energy, double tol, long long m, long long n, float* out,
                          cudaStream_t s) {
  k_probe_features<<<1, 32, 0, s>>>(mu, energy, tol, m, n, out);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

int launch_mlp_forward(const float* params, const float* x, int n, float* y, cudaStream_t s) {
  if (n <= 0) return TT_OK;
  k_mlp_forward<<<(n + 127) / 128, 128, 0, s>>>(params, x, n, y);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

int launch_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* t, int n, int steps,
                     int batch, float lr, int step0, unsigned long long seed, float* loss_trace, float* grad_out,
                     int mode, cudaStream_t s) {
  TT_TRY(train_attr());
  k_mlp_train<<<1, TT_THREADS, TRAIN_SMEM, s>>>(params, adam_m, adam_v, x, t, n, steps, batch, lr, step0, seed,
                                                  loss_trace, grad_out, mode);
  count_launch();
  TT_LAUNCH_CHECK();
  return TT_OK;
}

}  // namespace ttr
