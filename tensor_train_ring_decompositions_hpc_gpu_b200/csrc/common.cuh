// Shared helpers of the TT/TR-SVD kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "ttrsvd.h"

namespace ttr {

// Thread-local error message for tt_last_error().
void set_error(int code, const char* fmt, ...);

#define TT_TRY(expr)                  \
  do {                                \
    int st_ = (expr);                 \
    if (st_ != TT_OK) return st_;     \
  } while (0)

#define TT_CUDA(expr)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (expr);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      ::ttr::set_error(TT_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr,            \
                       cudaGetErrorString(e_));                                           \
      return TT_ERR_CUDA;                                                                 \
    }                                                                                     \
  } while (0)

#define TT_LAUNCH_CHECK()                                                                 \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      ::ttr::set_error(TT_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,               \
                       cudaGetErrorString(e_));                                           \
      return TT_ERR_CUDA;                                                                 \
    }                                                                                     \
  } while (0)

// Device status word written by kernels whose work can fail (non-convergence, timeouts).
struct DevStatus {
  int code;     // tt_status of the first failure, 0 if none
  int detail;   // kernel-specific detail (sweeps used, stage index, ...)
  int sweeps;   // largest Jacobi sweep count seen
  int pad;
};

__device__ __forceinline__ void dev_fail(DevStatus* st, int code, int detail) {
  if (st) {
    if (atomicCAS(&st->code, 0, code) == 0) st->detail = detail;
  }
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
inline long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

// Current device, its multiprocessor count (cached per device), and a once-per-device raise
// of a kernel's dynamic shared-memory limit (cudaFuncSetAttribute acts on the current device
// only).  smem_optin returns TT_OK or TT_ERR_CUDA with the error message set.
int cur_device();
int dev_sms();
int dev_smem_max();  // opt-in shared memory per block of the current device
int smem_optin(const void* fn, size_t bytes);
template <typename K>
inline int smem_optin_k(K* kernel, size_t bytes) {
  return smem_optin(reinterpret_cast<const void*>(kernel), bytes);
}

// Paired FP32 FMA (fma.rn.f32x2: two lanes of an FP32 pair per issue slot, each rounded like
// fmaf) and the moves in and out of a pair.
__device__ __forceinline__ uint64_t f2_dup(float a) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void ffma2(uint64_t& d, uint64_t a, uint64_t b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

// Launch-count accounting (kernels launched by the current library call).
extern thread_local int g_kernel_launches;
inline void count_launch(int n = 1) { g_kernel_launches += n; }

}  // namespace ttr
