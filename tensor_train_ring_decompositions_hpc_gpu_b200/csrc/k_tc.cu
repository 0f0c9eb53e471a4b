// tcgen05 / TMA tensor-core GEMM engine (placeholder until the kernels land).
#include "kernels.cuh"

namespace ttr {
bool tc_available() { return false; }
int launch_sketch_tc(const float*, long long, long long, const float*, int, long long, long long,
                     double*, Arena&, cudaStream_t) {
  return TT_ERR_UNSUPPORTED;
}
int launch_project_tc(const float*, long long, long long, const float*, int, long long, float*,
                      long long, int, int, int, Arena&, cudaStream_t) {
  return TT_ERR_UNSUPPORTED;
}
}  // namespace ttr
