// Allocation-free sketch entry point: tt_k_sketch_noalloc.
//
// Who needs it: callers that must not call cudaMalloc at all -- a process whose device
// memory is owned by another allocator (a framework's caching allocator or an arena reserved
// at start-up, where a raw cudaMalloc would break the budget or fail because the memory is
// already taken), and latency-critical loops where cudaMalloc/cudaFree are not acceptable
// because they can synchronise the device.  Such callers cannot create a tt_ctx (its
// workspace is allocated), so this entry point takes no context: the inputs and the output
// are the caller's, and the split-K scratch of the sketch kernel lives in one file-scope
// static device array that every GPU loading the library holds until the process exits.
//
// Limits and sharing rules:
//  * the scratch holds kScratchDoubles FP64 values (16 MiB per device); m * N must fit, and
//    the number of column splits is lowered until all partial sums fit;
//  * every call uses the same array and leaves its partial sums there; the device status word
//    at its start is cleared by each call, the partial sums are fully overwritten;
//  * calls whose work overlaps on the GPU (other streams, other host threads) race on the
//    array and give wrong results: serialise them;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress,
//    with that device current) and sets the kernels' shared-memory attributes; make that first
//    call before any stream capture.
#include <mutex>

#include "kernels.cuh"

namespace {

constexpr long long kScratchDoubles = 1LL << 21;  // 16 MiB
constexpr long long kStatusDoubles = 32;          // 256 B: status word, keeps partials 256-B aligned
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_sketch_scratch[kScratchDoubles];

std::mutex g_setup_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_sketch_scratch on the current device (looked up once per device).
int scratch_address(double** out) {
  int dev = 0;
  TT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    ttr::set_error(TT_ERR_UNSUPPORTED, "device %d beyond the %d devices the static scratch covers", dev,
                   kMaxDevices);
    return TT_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_sketch_scratch);
    if (e != cudaSuccess || !ptr) {
      ttr::set_error(TT_ERR_CUDA, "cudaGetSymbolAddress of the sketch scratch: %s", cudaGetErrorString(e));
      return TT_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_addr[dev];
  return TT_OK;
}

}  // namespace

extern "C" int tt_k_sketch_noalloc(const float* a, long long m, long long n, const float* w, int N,
                                   long long ldw, double* y, int gemm, void* stream) {
  if (!a || !w || !y) {
    ttr::set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  if (gemm < TT_GEMM_AUTO || gemm > TT_GEMM_FP32) {
    ttr::set_error(TT_ERR_ARG, "gemm option %d (expected TT_GEMM_AUTO, TT_GEMM_TC or TT_GEMM_FP32)", gemm);
    return TT_ERR_ARG;
  }
  if (m < 1 || n < 1 || N < 1 || N > TT_MAX_SMALL || ldw < n) {
    ttr::set_error(TT_ERR_SHAPE, "sketch shape m=%lld n=%lld N=%d ldw=%lld", m, n, N, ldw);
    return TT_ERR_SHAPE;
  }
  const long long cap = kScratchDoubles - kStatusDoubles;
  if ((double)m * (double)N > (double)cap) {
    ttr::set_error(TT_ERR_SHAPE,
                   "m * N = %lld * %d exceeds the %lld-double static scratch of tt_k_sketch_noalloc", m, N, cap);
    return TT_ERR_SHAPE;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (s) {
    // The scratch address below belongs to the current device; a stream of another device
    // would hand its kernels a pointer they cannot use.
    int cur = 0, sdev = 0;
    TT_CUDA(cudaGetDevice(&cur));
    TT_CUDA(cudaStreamGetDevice(s, &sdev));
    if (sdev != cur) {
      ttr::set_error(TT_ERR_ARG, "stream belongs to device %d but device %d is current", sdev, cur);
      return TT_ERR_ARG;
    }
  }
  double* base = nullptr;
  TT_TRY(scratch_address(&base));
  ttr::DevStatus* st = reinterpret_cast<ttr::DevStatus*>(base);
  double* part = base + kStatusDoubles;
  TT_CUDA(cudaMemsetAsync(st, 0, sizeof(ttr::DevStatus), s));
  int rc = TT_ERR_UNSUPPORTED;
  if (gemm != TT_GEMM_FP32 && ttr::tc_available())
    rc = ttr::launch_sketch_tc_static(a, m, n, w, N, 1, ldw, y, part, (size_t)cap, st, s);
  if (rc == TT_ERR_UNSUPPORTED)
    rc = ttr::launch_sketch_simt_static(a, m, n, w, N, 1, ldw, y, part, (size_t)cap, s);
  TT_TRY(rc);
  ttr::DevStatus h{};
  TT_CUDA(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
  TT_CUDA(cudaStreamSynchronize(s));
  if (h.code) {
    ttr::set_error(h.code, "device status %d (detail %d)", h.code, h.detail);
    return h.code;
  }
  return TT_OK;
}
