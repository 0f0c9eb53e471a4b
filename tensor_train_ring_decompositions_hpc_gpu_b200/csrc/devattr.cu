// Per-device launch attributes.  cudaFuncSetAttribute and the multiprocessor count belong to
// the device that is current when they are queried, and one process may drive several
// devices (one context per device), so both are cached per device here instead of once per
// process.
#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace ttr {
namespace {
std::mutex g_attr_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_set;  // (device, kernel) -> bytes raised to
constexpr int kMaxDev = 64;
int g_dev_sms[kMaxDev] = {0};
int g_dev_smem[kMaxDev] = {0};
}  // namespace

int cur_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return dev;
}

int dev_sms() {
  const int dev = cur_device();
  if (dev >= 0 && dev < kMaxDev && g_dev_sms[dev] > 0) return g_dev_sms[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    n = 148;
  }
  if (dev >= 0 && dev < kMaxDev) g_dev_sms[dev] = n;
  return n;
}

int dev_smem_max() {
  const int dev = cur_device();
  if (dev >= 0 && dev < kMaxDev && g_dev_smem[dev] > 0) return g_dev_smem[dev];
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0) {
    cudaGetLastError();
    v = 48 * 1024;
  }
  if (dev >= 0 && dev < kMaxDev) g_dev_smem[dev] = v;
  return v;
}

int smem_optin(const void* fn, size_t bytes) {
  const int dev = cur_device();
  std::lock_guard<std::mutex> lk(g_attr_mu);
  auto key = std::make_pair(dev, fn);
  auto it = g_smem_set.find(key);
  if (it != g_smem_set.end() && it->second >= bytes) return TT_OK;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(TT_ERR_CUDA, "shared-memory attribute (%zu bytes) refused on device %d", bytes, dev);
    return TT_ERR_CUDA;
  }
  g_smem_set[key] = bytes;
  return TT_OK;
}

}  // namespace ttr
