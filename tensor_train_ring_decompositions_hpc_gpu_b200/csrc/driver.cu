// Host side of the TT-SVD / TR-SVD chain: context, workspace planning, the per-unfolding
// factorisation (exact Gram-eigen or randomized EDrSVD) and the C ABI of ttrsvd.h.
//
// Chain (reference TT6:799-958 / TR6:827-1004): unfolding j is the column-major
// (r_{j-1} n_j) x rest matrix; after step j the projected factor is re-read in place as the
// next unfolding.  Steps whose target rank equals the row count (no truncation) are
// carried as a pending orthogonal rotation P instead of being rewritten: the true data is
// P^T times the raw data, every later quantity computed from the raw data is unchanged
// except the next core, which gets the block rotation (I (x) P^T) folded in.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace ttr {

static thread_local char g_err[512] = "";
void set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int n = snprintf(g_err, sizeof(g_err), "[%d] ", code);
  if (n < 0) n = 0;
  vsnprintf(g_err + n, sizeof(g_err) - n, fmt, ap);
  va_end(ap);
}

}  // namespace ttr

using namespace ttr;

struct tt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  char* arena = nullptr;
  size_t cap = 0;
  DevStatus* dstat = nullptr;
  DevStatus* hstat = nullptr;
  double* dsig = nullptr;  // TT_MAX_ORDER x TT_STATS_MAX_SIGMA
  double* hsig = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> pool;  // per-pass timing events (TT_FLAG_PROFILE)
  float* pred = nullptr;          // predictor parameters, then features (8) and outputs (3)
  size_t chunk_bytes = 256ull << 20;  // host-streaming chunk
  cudaStream_t copy_stream = nullptr;  // host-streaming copies
  cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_used[2] = {nullptr, nullptr};
  cudaStream_t side_stream = nullptr;  // eigen-solve of a folded step, overlapped with the next step
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  size_t alloc_limit = 0;  // workspace bytes above which growth fails with TT_ERR_NOMEM (0: none)
};

extern "C" const char* tt_last_error(void) { return ttr::g_err; }
extern "C" int tt_abi_version(void) { return TTRSVD_ABI_VERSION; }

extern "C" void tt_default_opts(tt_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->method = TT_METHOD_EDRSVD;
  o->gemm = TT_GEMM_AUTO;
  o->oversample = 8;
  o->power_iters = 0;
  o->seed = 1234ULL;
  o->eps = 0.0;
  o->flags = TT_FLAG_KEEP_SIGMA;
  o->max_sweeps = 40;
}

extern "C" int tt_ctx_create(tt_ctx** out, int device, void* stream) {
  if (!out) {
    set_error(TT_ERR_ARG, "null ctx pointer");
    return TT_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  TT_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error(TT_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    return TT_ERR_ARG;
  }
  TT_CUDA(cudaSetDevice(device));
  int major = 0;
  TT_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major != 10) {
    set_error(TT_ERR_UNSUPPORTED, "libttrsvd is built for sm_100a; device %d has compute capability %d.x",
              device, major);
    return TT_ERR_UNSUPPORTED;
  }
  tt_ctx* c = new tt_ctx();
  c->device = device;
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMalloc(&c->dstat, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&c->hstat, sizeof(DevStatus)) != cudaSuccess ||
      cudaMalloc(&c->dsig, sizeof(double) * TT_MAX_ORDER * TT_STATS_MAX_SIGMA) != cudaSuccess ||
      cudaMallocHost(&c->hsig, sizeof(double) * TT_MAX_ORDER * TT_STATS_MAX_SIGMA) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    set_error(TT_ERR_NOMEM, "context allocation failed");
    tt_ctx_destroy(c);
    return TT_ERR_NOMEM;
  }
  *out = c;
  return TT_OK;
}

extern "C" int tt_ctx_destroy(tt_ctx* c) {
  if (!c) return TT_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->arena) cudaFree(c->arena);
  if (c->dstat) cudaFree(c->dstat);
  if (c->hstat) cudaFreeHost(c->hstat);
  if (c->dsig) cudaFree(c->dsig);
  if (c->hsig) cudaFreeHost(c->hsig);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
  if (c->pred) cudaFree(c->pred);
  for (int b = 0; b < 2; ++b) {
    if (c->ev_copied[b]) cudaEventDestroy(c->ev_copied[b]);
    if (c->ev_used[b]) cudaEventDestroy(c->ev_used[b]);
  }
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->side_stream) cudaStreamDestroy(c->side_stream);
  delete c;
  return TT_OK;
}

extern "C" int tt_ctx_set_stream(tt_ctx* c, void* stream) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  return TT_OK;
}

extern "C" int tt_ctx_set_predictor(tt_ctx* c, const float* params) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  TT_CUDA(cudaSetDevice(c->device));
  if (!params) {
    if (c->pred) {
      if (c->stream) TT_CUDA(cudaStreamSynchronize(c->stream));
      cudaFree(c->pred);
    }
    c->pred = nullptr;
    return TT_OK;
  }
  if (!c->pred && cudaMalloc(&c->pred, sizeof(float) * (TT_MLP_PARAMS + 16)) != cudaSuccess) {
    c->pred = nullptr;
    set_error(TT_ERR_NOMEM, "predictor allocation");
    return TT_ERR_NOMEM;
  }
  TT_CUDA(cudaMemcpyAsync(c->pred, params, sizeof(float) * TT_MLP_PARAMS, cudaMemcpyHostToDevice, c->stream));
  TT_CUDA(cudaStreamSynchronize(c->stream));
  return TT_OK;
}

extern "C" int tt_ctx_set_stream_chunk(tt_ctx* c, size_t bytes) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  c->chunk_bytes = bytes;
  return TT_OK;
}

extern "C" int tt_ctx_set_alloc_limit(tt_ctx* c, size_t bytes) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  c->alloc_limit = bytes;
  return TT_OK;
}

extern "C" int tt_ctx_reserve(tt_ctx* c, size_t bytes) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  if (bytes <= c->cap) return TT_OK;
  if (c->alloc_limit && bytes > c->alloc_limit) {
    set_error(TT_ERR_NOMEM, "workspace of %zu bytes above the context's allocation limit of %zu bytes", bytes,
              c->alloc_limit);
    return TT_ERR_NOMEM;
  }
  TT_CUDA(cudaSetDevice(c->device));
  if (c->arena) {
    TT_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(c->arena);
    c->arena = nullptr;
    c->cap = 0;
  }
  bytes = (bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1);
  if (cudaMalloc(&c->arena, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(TT_ERR_NOMEM, "workspace of %zu bytes", bytes);
    return TT_ERR_NOMEM;
  }
  c->cap = bytes;
  return TT_OK;
}

namespace {

enum Path { PATH_EXACT_ROWS = 0, PATH_EXACT_COLS = 1, PATH_RAND = 2, PATH_IDENTITY = 3 };

// Internal option bit (above the public TT_FLAG_* range): adaptive ranks may fold a step whose
// chosen rank keeps every row.
constexpr int kFlagAdaptiveFold = 1 << 30;

struct Step {
  long long m = 0, cols = 0;
  int r_req = 0, r_eff = 0, ks = 0;
  int path = PATH_EXACT_ROWS;
  bool fold = false;     // full-rank step carried as a pending rotation
  bool perm231 = false;  // TR step 1
  long long next_elems = 0;
  // Row compaction: a basis zero-padded beyond r_eff produces zero rows in the next data, so
  // only the first n_out rows are written and later unfoldings skip them; the cores get the
  // zero rows back.  rows_in = rows of the stored data per mode index entering this step,
  // core_rows = the core's first rank; n_out = rows written; r1_out = TR bond r1 actually
  // carried after step 1 (n_out = r0 * r1_out).
  int rows_in = 1, core_rows = 1, n_out = 0, r1_out = 0;
};

struct Plan {
  int d = 0;
  bool ring = false;
  std::vector<long long> n;
  std::vector<int> r;
  std::vector<Step> steps;
  long long total = 0;
  size_t max_data = 0, max_omega = 0, max_y = 0, max_y0 = 0, max_bt = 0, max_core = 0, max_ws = 0;
  size_t max_ef = (size_t)TT_MAX_SMALL * TT_MAX_SMALL;  // FP32 basis (m x r or ks x r)
  int max_small = 0;
  int last_rows = 1;  // rows per mode index of the data left for the last core
  long long stream_cols = 0;  // host streaming: columns of the first unfolding per chunk (0: off)
};

// An exact step whose Gram comes from the tensor cores (more than 32 rows) and that truncates
// gets its kept subspace refined by exact Rayleigh-Ritz (see run_chain); b = r + 16 columns.
bool refine_exact(const Step& st, int engine, bool adaptive) {
  return st.path == PATH_EXACT_ROWS && engine == TT_GEMM_TC && !adaptive && st.m > 32 && st.r_eff < st.m &&
         !st.perm231;
}
int refine_width(const Step& st) { return (int)std::min<long long>(st.m, (long long)st.r_eff + 16); }

int engine_of(const tt_opts& o) {
  if (o.gemm == TT_GEMM_FP32) return TT_GEMM_FP32;
  return tc_available() ? TT_GEMM_TC : TT_GEMM_FP32;
}

// Engine of a bulk pass over an m x cols unfolding.  TT_GEMM_AUTO keeps passes below 2^24
// elements on the FP32 kernels (they are cheap there and carry full FP32 precision); the
// tensor cores take the large unfoldings, where HBM bandwidth decides.
int engine_for(const tt_opts& o, long long m, long long cols) {
  const int e = engine_of(o);
  if (e == TT_GEMM_TC && o.gemm == TT_GEMM_AUTO && (double)m * (double)cols < 16777216.0)
    return TT_GEMM_FP32;
  return e;
}

struct Step;
bool refine_exact(const Step& st, int engine, bool adaptive);
int refine_width(const Step& st);

int make_plan(int d, const int* n, const int* r, bool ring, const tt_opts& o, Plan& P) {
  if (d < 2 || d > TT_MAX_ORDER) {
    set_error(TT_ERR_SHAPE, "order %d outside [2, %d]", d, TT_MAX_ORDER);
    return TT_ERR_SHAPE;
  }
  if (!n || !r) {
    set_error(TT_ERR_ARG, "null mode or rank array");
    return TT_ERR_ARG;
  }
  P.d = d;
  P.ring = ring;
  P.n.assign(n, n + d);
  P.r.assign(r, r + d + 1);
  P.total = 1;
  for (int k = 0; k < d; ++k) {
    if (n[k] < 1) {
      set_error(TT_ERR_SHAPE, "mode size n[%d] = %d", k, n[k]);
      return TT_ERR_SHAPE;
    }
    P.total *= n[k];
  }
  for (int k = 0; k <= d; ++k)
    if (r[k] < 1) {
      set_error(TT_ERR_RANK, "rank r[%d] = %d", k, r[k]);
      return TT_ERR_RANK;
    }
  if (!ring && (r[0] != 1 || r[d] != 1)) {
    set_error(TT_ERR_RANK, "TT ranks need r[0] = r[d] = 1 (got %d, %d)", r[0], r[d]);
    return TT_ERR_RANK;
  }
  if (ring && r[0] != r[d]) {
    set_error(TT_ERR_RANK, "ring ranks need r[0] = r[d] (got %d, %d)", r[0], r[d]);
    return TT_ERR_RANK;
  }
  const int s = std::max(0, o.oversample);
  const bool nofold = (o.flags & TT_FLAG_NO_FOLD) != 0;
  long long size = P.total;  // elements of the current (raw) data
  long long rows_prev = 1;   // rows per mode index of the stored data (effective r_{k-1})
  P.steps.clear();
  for (int k = 0; k < d - 1; ++k) {
    Step st;
    const bool first_ring = ring && k == 0;
    st.m = first_ring ? n[0] : rows_prev * n[k];
    st.cols = size / st.m;
    st.r_req = first_ring ? r[0] * r[1] : r[k + 1];
    st.perm231 = first_ring && r[0] > 1;
    const long long mn = std::min(st.m, st.cols);
    st.r_eff = (int)std::min<long long>(st.r_req, mn);
    // Exact Gram-eigen step when the small side is tiny (<= 64: one-CTA eigen-solver), when
    // a sketch would cover half of it anyway, or on request; otherwise EDrSVD.
    const bool small_exact =
        mn <= 64 || (mn <= TT_MAX_SMALL && 2LL * (st.r_eff + s) >= mn);
    if (o.method == TT_METHOD_EXACT || small_exact) {
      if (mn > TT_MAX_SMALL) {
        set_error(TT_ERR_UNSUPPORTED, "exact step %d needs min(m, n) = %lld <= %d", k, mn, TT_MAX_SMALL);
        return TT_ERR_UNSUPPORTED;
      }
      st.path = (st.m <= st.cols) ? PATH_EXACT_ROWS : PATH_EXACT_COLS;
      st.ks = (int)mn;
    } else {
      st.path = PATH_RAND;
      // The learned form may pick oversampling up to TT_LEARNED_MAX_S: its sketch width limit
      // makes room for that.
      const int s_cap = (o.flags & TT_FLAG_LEARNED) ? std::max(s, TT_LEARNED_MAX_S) : s;
      st.ks = (int)std::min<long long>({(long long)st.r_eff + s_cap, mn, (long long)TT_MAX_SMALL});
      if (st.ks < st.r_eff) {
        set_error(TT_ERR_UNSUPPORTED, "step %d: rank %d above the sketch limit %d", k, st.r_eff, TT_MAX_SMALL);
        return TT_ERR_UNSUPPORTED;
      }
    }
    st.fold = !nofold && !st.perm231 && st.path == PATH_EXACT_ROWS && st.r_req == st.m &&
              st.r_eff == st.m && !(ring && k == 0) && rows_prev == r[k];
    if (st.fold && (o.flags & TT_FLAG_IDENTITY_GAUGE)) st.path = PATH_IDENTITY;
    st.rows_in = first_ring ? 1 : (int)rows_prev;
    st.core_rows = first_ring ? 1 : r[k];
    if (first_ring) {
      st.r1_out = (st.r_eff + r[0] - 1) / r[0];
      st.n_out = r[0] * st.r1_out;
    } else {
      st.r1_out = 0;
      st.n_out = st.fold ? st.r_req : st.r_eff;
    }
    st.next_elems = (long long)st.n_out * st.cols;
    P.steps.push_back(st);
    size = st.fold ? size : st.next_elems;
    rows_prev = first_ring ? st.r1_out : st.n_out;
    P.last_rows = (int)rows_prev;
    if (st.perm231 && st.path == PATH_EXACT_COLS)
      P.max_bt = std::max<size_t>(P.max_bt, (size_t)st.next_elems);
    if (!st.fold) P.max_data = std::max<size_t>(P.max_data, (size_t)st.next_elems);
    if (st.path == PATH_EXACT_ROWS && st.m > 32 && st.r_eff < st.m && !st.perm231) {
      // room for a refined exact step (U0: m x b, Z: cols x b)
      const int b = refine_width(st);
      P.max_y = std::max<size_t>(P.max_y, (size_t)st.m * b);
      P.max_bt = std::max<size_t>(P.max_bt, (size_t)st.cols * b);
      P.max_ws = std::max(P.max_ws, project_ws_bytes(st.m, st.cols, b));
      P.max_ws = std::max(P.max_ws, project_ws_bytes(b, st.cols, st.r_req));
      P.max_ws = std::max(P.max_ws, gram_ws_bytes(st.cols, b));
    }
    P.max_core = std::max<size_t>(P.max_core, (size_t)st.m * std::max(st.r_req, st.ks));
    P.max_ef = std::max<size_t>(P.max_ef, (size_t)std::max<long long>(st.m, st.ks) * st.r_req);
    P.max_small = std::max(P.max_small, std::max(st.ks, (int)std::min<long long>(mn, TT_MAX_SMALL)));
    if (st.path == PATH_RAND) {
      P.max_omega = std::max<size_t>(P.max_omega, (size_t)st.cols * st.ks);
      P.max_y = std::max<size_t>(P.max_y, (size_t)st.m * std::max(st.ks, TT_PROBE_COLS));
      if (o.flags & TT_FLAG_LEARNED) P.max_y0 = std::max<size_t>(P.max_y0, (size_t)st.m * TT_PROBE_COLS);
      P.max_bt = std::max<size_t>(P.max_bt, (size_t)st.cols * st.ks);
      // the adaptive modes run narrower sketches (and the probe) within the same buffers
      const bool narrow = (o.flags & (TT_FLAG_ADAPTIVE_KS | TT_FLAG_LEARNED)) != 0;
      for (int w = narrow ? 1 : st.ks; w <= st.ks; ++w) {
        P.max_ws = std::max(P.max_ws, sketch_ws_bytes(st.m, st.cols, w));
        P.max_ws = std::max(P.max_ws, gram_ws_bytes(st.cols, w));
        P.max_ws = std::max(P.max_ws, gram_ws_bytes(st.m, w));
        P.max_ws = std::max(P.max_ws, gram_tc_ws_bytes(w, st.cols));
        P.max_ws = std::max(P.max_ws, gram32x_ws_bytes());
        P.max_ws = std::max(P.max_ws, project_ws_bytes(st.m, st.cols, w));
        P.max_ws = std::max(P.max_ws, project_ws_bytes(w, st.cols, std::min(w, st.r_req)));
      }
      P.max_ws = std::max(P.max_ws, project_ws_bytes(st.ks, st.cols, st.r_req));
      P.max_ws = std::max(P.max_ws, syev_ws_bytes(st.ks, o.max_sweeps));
    } else {
      P.max_ws = std::max(P.max_ws, project_ws_bytes(st.m, st.cols, st.r_req));
      P.max_ws = std::max(P.max_ws, gram_ws_bytes(std::max(st.m, st.cols), (int)mn));
      P.max_ws = std::max(P.max_ws, gram_tc_ws_bytes(st.m, st.cols));
      P.max_ws = std::max(P.max_ws, gram32x_ws_bytes());
      P.max_ws = std::max(P.max_ws, syev_ws_bytes((int)mn, o.max_sweeps));
    }
  }
  P.max_ws += (size_t)TT_MAX_SMALL * TT_MAX_SMALL * sizeof(double) * 8;
  return TT_OK;
}

size_t core_elems(const Plan& P, int k) { return (size_t)P.r[k] * P.n[k] * P.r[k + 1]; }

struct Bufs {
  float* x = nullptr;        // input on device
  float* data[2] = {nullptr, nullptr};
  float* omega = nullptr;
  double* yd = nullptr;
  float* yf = nullptr;
  double* y0 = nullptr;     // learned probe Y0 (m x TT_PROBE_COLS, FP64)
  double* resid = nullptr;  // per probe column ||(I - QQ^T) y0_j||^2
  float* bt = nullptr;
  float* corebuf = nullptr;
  float* ef = nullptr;
  double* w = nullptr;
  double* evals = nullptr;
  double* evecs = nullptr;
  double* colscale = nullptr;
  double* pend[2] = {nullptr, nullptr};
  int* flag = nullptr;
  std::vector<float*> cores;  // device cores
  float* chunk[2] = {nullptr, nullptr};  // host streaming
  double* wacc = nullptr;
  double* w2 = nullptr;       // folded step: Gram, eigenpairs and basis on the side stream
  double* evals2 = nullptr;
  double* evecs2 = nullptr;
  float* ef2 = nullptr;
};

size_t plan_bytes(const Plan& P, bool host_io) {
  const size_t S = TT_MAX_SMALL;
  size_t b = 0;
  auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
  if (host_io && !P.stream_cols) add(P.total * sizeof(float));
  if (P.stream_cols) {
    add((size_t)P.steps[0].m * P.stream_cols * sizeof(float) * 2);
    add(S * S * sizeof(double));
  }
  add(P.max_data * sizeof(float));
  add(P.max_data * sizeof(float));
  add(P.max_omega * sizeof(float));
  add(P.max_y * sizeof(double));
  add(P.max_y * sizeof(float));
  add(P.max_y0 * sizeof(double));
  add(TT_PROBE_COLS * sizeof(double));
  add(P.max_bt * sizeof(float));
  add(P.max_core * sizeof(float));
  add(P.max_ef * sizeof(float));
  add(S * S * sizeof(double) * 4);
  add(S * sizeof(double) * 2);
  add(S * S * sizeof(double) * 2);
  add(256);
  add(S * S * sizeof(double) * 2 + S * sizeof(double) + 1024);  // side-stream eigen-solve
  add(P.max_ef * sizeof(float));
  if (host_io)
    for (int k = 0; k < P.d; ++k) add(core_elems(P, k) * sizeof(float));
  add(P.max_ws);
  return b + (1 << 20);
}

int carve(tt_ctx* c, const Plan& P, bool host_io, Bufs& B, Arena& ws) {
  Arena a{c->arena, c->cap, 0};
  const size_t S = TT_MAX_SMALL;
  if (host_io && !P.stream_cols) B.x = a.take<float>(P.total);
  if (P.stream_cols) {
    B.chunk[0] = a.take<float>((size_t)P.steps[0].m * P.stream_cols);
    B.chunk[1] = a.take<float>((size_t)P.steps[0].m * P.stream_cols);
    B.wacc = a.take<double>(S * S);
    if (!B.chunk[1] || !B.wacc) {
      set_error(TT_ERR_NOMEM, "streaming buffers");
      return TT_ERR_NOMEM;
    }
  }
  B.data[0] = a.take<float>(std::max<size_t>(P.max_data, 1));
  B.data[1] = a.take<float>(std::max<size_t>(P.max_data, 1));
  B.omega = a.take<float>(std::max<size_t>(P.max_omega, 1));
  B.yd = a.take<double>(std::max<size_t>(P.max_y, 1));
  B.yf = a.take<float>(std::max<size_t>(P.max_y, 1));
  B.y0 = a.take<double>(std::max<size_t>(P.max_y0, 1));
  B.resid = a.take<double>(TT_PROBE_COLS);
  B.bt = a.take<float>(std::max<size_t>(P.max_bt, 1));
  B.corebuf = a.take<float>(std::max<size_t>(P.max_core, 1));
  B.ef = a.take<float>(P.max_ef);
  B.w = a.take<double>(S * S);
  B.evecs = a.take<double>(S * S);
  B.pend[0] = a.take<double>(S * S);
  B.pend[1] = a.take<double>(S * S);
  B.evals = a.take<double>(S);
  B.colscale = a.take<double>(S);
  B.flag = a.take<int>(64);
  B.w2 = a.take<double>(S * S);
  B.evals2 = a.take<double>(S);
  B.evecs2 = a.take<double>(S * S);
  B.ef2 = a.take<float>(P.max_ef);
  if (host_io) {
    B.cores.resize(P.d);
    for (int k = 0; k < P.d; ++k) B.cores[k] = a.take<float>(core_elems(P, k));
  }
  if (!B.data[1] || !B.flag || !B.ef2 || (host_io && !B.cores[P.d - 1])) {
    set_error(TT_ERR_NOMEM, "workspace carve");
    return TT_ERR_NOMEM;
  }
  ws = Arena{c->arena + a.off, c->cap - a.off, 0};
  return TT_OK;
}

// Store sqrt(evals[0:cnt]) of step k for the stats (device-side copy; read back at the end).
__global__ void k_store_sigma(const double* evals, int cnt, double* dst) {
  const int i = threadIdx.x;
  if (i < TT_STATS_MAX_SIGMA) dst[i] = (i < cnt) ? sqrt(fmax(evals[i], 0.0)) : -1.0;
}

// Core (Rcore, ni, ncols) from the basis `raw` ((Rin ni) x ncols): a pending rotation is folded
// in (then Rin == Rcore), compacted rows Rin < Rcore come back as zero rows.
int emit_core(const float* raw, float* out, const double* pend, int Rin, int Rcore, long long ni, int ncols,
              cudaStream_t s) {
  if (pend) return launch_fold_rows(raw, out, pend, Rin, ni, ncols, s);
  if (Rin != Rcore) return launch_expand_rows(raw, Rin, out, Rcore, ni * ncols, s);
  TT_CUDA(cudaMemcpyAsync(out, raw, sizeof(float) * (size_t)Rin * ni * ncols, cudaMemcpyDeviceToDevice, s));
  return TT_OK;
}

__global__ void k_eye(double* p, int m) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < m * m) p[idx] = (idx % m == idx / m) ? 1.0 : 0.0;
}

// Accounting of the bulk passes: algorithmic FLOPs/bytes always, device time when profiling.
struct PassRec {
  int kind;
  int step;
  double bytes;
  cudaEvent_t a, b;
};
struct Passes {
  tt_ctx* c = nullptr;
  cudaStream_t s = nullptr;
  bool on = false;
  int cur_step = 0;
  size_t next = 0;
  double flops = 0.0, bytes = 0.0;
  std::vector<PassRec> recs;
  template <typename F>
  int run(int kind, double fl, double by, F&& fn) {
    flops += fl;
    bytes += by;
    cudaEvent_t a = nullptr, b = nullptr;
    if (on) {
      while (c->pool.size() < next + 2) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) break;
        c->pool.push_back(e);
      }
      if (c->pool.size() >= next + 2) {
        a = c->pool[next];
        b = c->pool[next + 1];
        next += 2;
        cudaEventRecord(a, s);
      }
    }
    const int st = fn();
    if (a) {
      cudaEventRecord(b, s);
      recs.push_back({kind, cur_step, by, a, b});
    }
    return st;
  }
};

__global__ void k_add_f64(const double* __restrict__ a, double* __restrict__ acc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] += a[i];
}

int run_chain(tt_ctx* c, const float* x_in, Plan P, const tt_opts& o, float* const* cores_out,
              tt_stats* stats) {
  const bool host_io = (o.flags & TT_FLAG_HOST_IO) != 0;
  TT_CUDA(cudaSetDevice(c->device));
  // a side-stream job of an earlier call that failed midway must not outlive its buffers
  if (c->side_stream) TT_CUDA(cudaStreamSynchronize(c->side_stream));
  TT_TRY(tt_ctx_reserve(c, plan_bytes(P, host_io)));
  Bufs B;
  Arena ws;
  TT_TRY(carve(c, P, host_io, B, ws));
  cudaStream_t s = c->stream;
  const int max_sweeps = o.max_sweeps > 0 ? o.max_sweeps : 40;
  g_kernel_launches = 0;
  Passes pass;
  pass.c = c;
  pass.s = s;
  pass.on = (o.flags & TT_FLAG_PROFILE) != 0;

  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), s));
  TT_CUDA(cudaEventRecord(c->ev0, s));
  const float* x = x_in;
  const bool stream = P.stream_cols > 0;  // x stays on the host; step 0 streams it
  if (host_io && !stream) {
    TT_CUDA(cudaMemcpyAsync(B.x, x_in, sizeof(float) * P.total, cudaMemcpyHostToDevice, s));
    x = B.x;
  }
  // One pass over the host-resident first unfolding: chunk ch (stream_cols columns) is copied
  // on the copy stream into buffer ch & 1 while the kernels of chunk ch - 1 run on s; fn(chunk,
  // first column, columns) enqueues a chunk's kernels on s.
  auto stream_pass = [&](auto&& fn) -> int {
    const long long m0 = P.steps[0].m, cols0 = P.steps[0].cols, cc = P.stream_cols;
    const long long nch = (cols0 + cc - 1) / cc;
    if (!c->copy_stream) {
      TT_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      for (int b = 0; b < 2; ++b) {
        TT_CUDA(cudaEventCreateWithFlags(&c->ev_copied[b], cudaEventDisableTiming));
        TT_CUDA(cudaEventCreateWithFlags(&c->ev_used[b], cudaEventDisableTiming));
      }
    }
    // buffers are free once the work already on s (an earlier pass) is done
    for (int b = 0; b < 2; ++b) TT_CUDA(cudaEventRecord(c->ev_used[b], s));
    auto issue = [&](long long ch) -> int {
      const int b = (int)(ch & 1);
      const long long c0 = ch * cc, nc = std::min(cc, cols0 - c0);
      TT_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_used[b], 0));
      TT_CUDA(cudaMemcpyAsync(B.chunk[b], x_in + c0 * m0, sizeof(float) * (size_t)(nc * m0), cudaMemcpyHostToDevice,
                              c->copy_stream));
      TT_CUDA(cudaEventRecord(c->ev_copied[b], c->copy_stream));
      return TT_OK;
    };
    TT_TRY(issue(0));
    if (nch > 1) TT_TRY(issue(1));
    for (long long ch = 0; ch < nch; ++ch) {
      const int b = (int)(ch & 1);
      const long long c0 = ch * cc, nc = std::min(cc, cols0 - c0);
      TT_CUDA(cudaStreamWaitEvent(s, c->ev_copied[b], 0));
      TT_TRY(fn((const float*)B.chunk[b], c0, nc));
      TT_CUDA(cudaEventRecord(c->ev_used[b], s));
      if (ch + 2 < nch) TT_TRY(issue(ch + 2));
    }
    return TT_OK;
  };
  std::vector<float*> cores(P.d);
  for (int k = 0; k < P.d; ++k) cores[k] = host_io ? B.cores[k] : cores_out[k];

  if (o.flags & TT_FLAG_CHECK_FINITE) {
    TT_CUDA(cudaMemsetAsync(B.flag, 0, sizeof(int), s));
    TT_TRY(launch_check_finite(x, P.total, B.flag, s));
    int hflag = 0;
    TT_CUDA(cudaMemcpyAsync(&hflag, B.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    TT_CUDA(cudaStreamSynchronize(s));
    if (hflag) {
      set_error(TT_ERR_NONFINITE, "input holds NaN or Inf");
      return TT_ERR_NONFINITE;
    }
  }

  // Adaptive ranks (o.eps > 0): delta-truncation of every unfolding, delta^2 = eps^2 ||X||^2 /
  // (d - 1) (the TT-SVD error bound); the caller's ranks are upper bounds.  Each decision reads
  // the eigenvalues back to the host, and the rest of the plan is rebuilt with the chosen rank.
  const bool adaptive = o.eps > 0.0;
  double delta2 = 0.0, energy = 0.0, xnorm2 = 0.0, tail_sum = 0.0;
  int eps_unmet = 0;  // steps whose rank bound left more than delta^2 discarded
  bool energy_exact = true;  // `energy` is exact (false after a step judged on the probe estimate)
  // A first step with an exact Gram of the whole tensor gives ||X||^2 as its eigenvalue sum
  // (the trace); otherwise one FP64 norm pass runs first.
  const bool norm_from_gram = adaptive && !P.steps.empty() && !stream &&
                              (P.steps[0].path == PATH_EXACT_ROWS || P.steps[0].path == PATH_EXACT_COLS);
  if (adaptive && !norm_from_gram) {
    const size_t mk = ws.mark();
    double* acc = ws.take<double>(2);
    if (!acc) {
      set_error(TT_ERR_NOMEM, "norm accumulator");
      return TT_ERR_NOMEM;
    }
    TT_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s));
    TT_TRY(launch_diff_norm(x, nullptr, P.total, acc, s));
    double h[2];
    TT_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
    TT_CUDA(cudaStreamSynchronize(s));
    ws.reset(mk);
    xnorm2 = h[1];
    energy = xnorm2;
    delta2 = o.eps * o.eps * xnorm2 / (double)(P.d - 1);
  }
  std::vector<int> rmax(P.r);  // caller's ranks (upper bounds in adaptive mode)
  tt_opts oplan = o;
  oplan.flags |= TT_FLAG_NO_FOLD;

  const float* cur = x;
  int slot = 0;
  const double* pend = nullptr;  // pending rotation (rows_in x rows_in), or null
  int pend_slot = 0;
  const int nsteps = (int)P.steps.size();
  // A folded exact step (full rank, rotation kept pending) does not change the data the next
  // step reads, so its eigen-solve, core and pending rotation run on a side stream while the
  // next step's bulk passes proceed; join_side() makes s wait before the rotation is used.
  bool side_pending = false;
  auto join_side = [&]() -> int {
    if (side_pending) {
      TT_CUDA(cudaStreamWaitEvent(s, c->ev_join, 0));
      side_pending = false;
    }
    return TT_OK;
  };
  // Gram of the rows of an unfolding with m <= 128 rows (the exact step).  Up to 32 rows: the
  // exact CUDA-core kernel in every form (FP32 products, FP64 sums), whose result resolves
  // eigenvalues down to ~1e-9 of the largest; the tensor cores' truncating FP32 accumulation
  // would bias the small ones.  Wider: tensor cores when allowed, else the FP32 engine.
  // `precise` (adaptive ranks: energies to ~1e-8 relative) keeps short unfoldings, whose few
  // partial sums do not average the FP32 rounding out, on FP64 products.
  auto gram_rows = [&](const float* a, long long mm, long long nc, double* w, int eng, bool precise) -> int {
    const bool long_unf = nc >= (1LL << 16);
    if (mm <= 32 && (!precise || long_unf)) {
      const int rc = launch_gram32x(a, nc, (int)mm, w, ws, c->dstat, s);
      if (rc != TT_ERR_UNSUPPORTED) return rc;
    }
    if (eng == TT_GEMM_TC && !precise) {
      const int rc = launch_gram_tc(a, mm, nc, w, ws, c->dstat, s);
      if (rc != TT_ERR_UNSUPPORTED) return rc;
    }
    return launch_gram(a, nc, (int)mm, mm, 1, w, precise && nc < (1LL << 22), ws, s);
  };
  int npasses = 0, natt = 0, nfall = 0;  // bulk passes, EDrSVD attempts, learned fallbacks
  std::vector<int> step_ks((size_t)nsteps, 0), step_pw((size_t)nsteps, 0), step_att((size_t)nsteps, 0);
  for (int k = 0; k < nsteps; ++k) {
    Step& st = P.steps[k];
    pass.cur_step = k;
    const int natt0 = natt;
    const long long m = st.m, cols = st.cols;
    int rq = st.r_req, re = st.r_eff;
    int nout = st.n_out;                            // rows of the next data (compacted)
    // Adaptive rank of this step from the first `nev` eigenvalues in B.evals: the smallest r
    // whose discarded energy, outside + sum_{i >= r} lambda_i, is <= delta^2.  `outside` is the
    // energy outside the eigen-decomposed subspace: 0 for an exact step (its Gram holds the whole
    // unfolding), the carried energy minus every eigenvalue for a plain EDrSVD attempt, and the
    // probe estimate for a learned attempt.
    // Eigenvalues of the attempt already read back with the probe estimate (learned steps: one
    // device round trip instead of two), or empty.
    std::vector<double> lam_pre;
    auto decide = [&](int nev, double outside) -> int {
      if (!adaptive) return TT_OK;
      std::vector<double> lam((size_t)nev);
      if (lam_pre.size() == (size_t)nev) {
        lam.swap(lam_pre);
      } else {
        TT_CUDA(cudaMemcpyAsync(lam.data(), B.evals, sizeof(double) * nev, cudaMemcpyDeviceToHost, s));
        TT_CUDA(cudaStreamSynchronize(s));
      }
      lam_pre.clear();
      double inside = 0.0;
      for (double v : lam) inside += std::max(v, 0.0);
      if (norm_from_gram && k == 0) {
        xnorm2 = inside;
        energy = xnorm2;
        delta2 = o.eps * o.eps * xnorm2 / (double)(P.d - 1);
      }
      const int cap = std::min(rmax[k + 1], std::min(nev, re));
      int r = 0;
      double tail = std::max(outside, 0.0) + inside, kept = 0.0;
      while (r < cap && (r == 0 || tail > delta2)) {
        const double l = std::max(lam[(size_t)r++], 0.0);
        tail -= l;
        kept += l;
      }
      tail = std::max(tail, 0.0);
      if (tail > delta2 * (1.0 + 1e-12)) ++eps_unmet;  // the bound stopped the truncation above delta
      tail_sum += tail;
      energy = kept;  // energy of the next data
      rq = re = nout = r;
      st.r_req = st.r_eff = st.n_out = r;
      st.next_elems = (long long)r * cols;
      P.r[k + 1] = r;
      Plan P2;
      const std::vector<int> nn(P.n.begin(), P.n.end());
      TT_TRY(make_plan(P.d, nn.data(), P.r.data(), P.ring, oplan, P2));
      for (size_t j = (size_t)k + 1; j < P.steps.size(); ++j) P.steps[j] = P2.steps[j];
      P.last_rows = P2.last_rows;
      return TT_OK;
    };
    const int pr1 = st.perm231 ? st.r1_out : 1;     // TR bond r1 carried after step 1
    const int rin = st.rows_in, rcore = st.core_rows;
    const int engine = engine_for(o, m, cols);
    float* next = B.data[slot];
    double* sigdst = c->dsig + (size_t)k * TT_STATS_MAX_SIGMA;
    const bool ring1 = P.ring && k == 0;
    float* core_dst = ring1 ? B.corebuf : cores[k];
    // For the ring's first core the (n1 x q) basis is rearranged below.
    const long long ni = P.n[k];

    if (st.path == PATH_IDENTITY) {
      // Core = (I (x) P^T) I_m as an (rows_in n_k) x m matrix; no pending rotation afterwards.
      k_eye<<<ceil_div(m * m, 256), 256, 0, s>>>(B.w, (int)m);
      count_launch();
      TT_LAUNCH_CHECK();
      if (pend) {
        TT_TRY(launch_f64_to_f32_cols(B.w, m, m, (int)m, B.corebuf, m, (int)m, s));
        TT_TRY(join_side());
        TT_TRY(launch_fold_rows(B.corebuf, core_dst, pend, rin, ni, (int)m, s));
      } else {
        TT_TRY(launch_f64_to_f32_cols(B.w, m, m, (int)m, core_dst, m, (int)m, s));
      }
      k_store_sigma<<<1, 64, 0, s>>>(B.evals, 0, sigdst);
      count_launch();
      pend = nullptr;
      continue;  // data unchanged
    }

    if (st.path == PATH_EXACT_ROWS && stream && k == 0) {
      // host-streamed first unfolding: Gram summed over the chunks in FP64, projection per chunk
      npasses += 2;
      TT_TRY(pass.run(TT_PASS_GRAM, 2.0 * m * m * cols, 4.0 * m * cols, [&]() -> int {
        TT_CUDA(cudaMemsetAsync(B.wacc, 0, sizeof(double) * m * m, s));
        TT_TRY(stream_pass([&](const float* a, long long, long long nc) -> int {
          TT_TRY(gram_rows(a, m, nc, B.w, engine_for(o, m, nc), false));
          k_add_f64<<<ceil_div(m * m, 256), 256, 0, s>>>(B.w, B.wacc, (int)(m * m));
          count_launch();
          TT_LAUNCH_CHECK();
          return TT_OK;
        }));
        TT_CUDA(cudaMemcpyAsync(B.w, B.wacc, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, s));
        return TT_OK;
      }));
      TT_TRY(launch_syev(B.w, (int)m, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
      k_store_sigma<<<1, 64, 0, s>>>(B.evals, (int)std::min<long long>(m, TT_STATS_MAX_SIGMA), sigdst);
      count_launch();
      TT_TRY(launch_f64_to_f32_cols(B.evecs, m, m, re, B.ef, m, rq, s));
      TT_TRY(launch_canon_cols(B.ef, m, re, m, B.evecs, (int)m, m, s));
      TT_TRY(join_side());
      TT_TRY(emit_core(B.ef, core_dst, pend, rin, rcore, ni, rq, s));
      TT_TRY(pass.run(TT_PASS_PROJECT, 2.0 * m * cols * nout, 4.0 * m * cols + 4.0 * nout * cols, [&]() -> int {
        return stream_pass([&](const float* a, long long c0, long long nc) -> int {
          return launch_project(a, m, nc, B.ef, nout, m, next + c0 * nout, nout, OUT_ROWMAJOR, 1, 1,
                                engine_for(o, m, nc), ws, c->dstat, s);
        });
      }));
    } else if (st.path == PATH_EXACT_ROWS && st.fold && !adaptive && m <= 64) {
      // folded step: Gram on s, the rest on the side stream (see join_side)
      npasses += 1;
      TT_TRY(join_side());  // one side job at a time: its buffers are reused here
      TT_TRY(pass.run(TT_PASS_GRAM, 2.0 * m * m * cols, 4.0 * m * cols,
                      [&] { return gram_rows(cur, m, cols, B.w2, engine, false); }));
      if (!c->side_stream) {
        TT_CUDA(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
        TT_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
        TT_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
      }
      cudaStream_t ss = c->side_stream;
      TT_CUDA(cudaEventRecord(c->ev_fork, s));
      TT_CUDA(cudaStreamWaitEvent(ss, c->ev_fork, 0));
      TT_TRY(launch_syev(B.w2, (int)m, B.evals2, B.evecs2, max_sweeps, ws, c->dstat, ss));
      k_store_sigma<<<1, 64, 0, ss>>>(B.evals2, (int)std::min<long long>(m, TT_STATS_MAX_SIGMA), sigdst);
      count_launch();
      TT_TRY(launch_f64_to_f32_cols(B.evecs2, m, m, re, B.ef2, m, rq, ss));
      TT_TRY(launch_canon_cols(B.ef2, m, re, m, B.evecs2, (int)m, m, ss));
      TT_TRY(emit_core(B.ef2, core_dst, pend, rin, rcore, ni, rq, ss));
      double* pnew = B.pend[pend_slot ^ 1];
      TT_CUDA(cudaMemcpyAsync(pnew, B.evecs2, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, ss));
      TT_CUDA(cudaEventRecord(c->ev_join, ss));
      side_pending = true;
      pend = pnew;
      pend_slot ^= 1;
      continue;
    } else if (st.path == PATH_EXACT_ROWS) {
      npasses += st.fold ? 1 : 2;
      TT_TRY(pass.run(TT_PASS_GRAM, 2.0 * m * m * cols, 4.0 * m * cols,
                      [&] { return gram_rows(cur, m, cols, B.w, engine, adaptive); }));
      // A step refined below reads only the span of the top b <= 32 eigenvectors, which the
      // exact Rayleigh-Ritz then corrects: above 64 rows the subspace solver gives it for a
      // fraction of the full solve.
      if (!st.fold && refine_exact(st, engine, adaptive) && m > 64 && refine_width(st) <= 32)
        TT_TRY(launch_syev_top(B.w, (int)m, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
      else
        TT_TRY(launch_syev(B.w, (int)m, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
      k_store_sigma<<<1, 64, 0, s>>>(B.evals, (int)std::min<long long>(m, TT_STATS_MAX_SIGMA), sigdst);
      count_launch();
      TT_TRY(decide((int)m, 0.0));
      energy_exact = true;
      // An adaptive rank that keeps every row makes the step a rotation: fold it like a
      // planned full-rank step (the next step's geometry is the same either way).
      const bool fold = st.fold || (adaptive && !ring1 && !st.perm231 && rq == m && re == m && rin == rcore &&
                                    (o.flags & kFlagAdaptiveFold));
      if (refine_exact(st, engine, adaptive) && !fold) {
        // Exact Rayleigh-Ritz on the span of the top b eigenvectors of the tensor-core Gram:
        // that Gram's TF32 rounding tilts eigenvectors of close eigenvalues (a flat spectrum
        // around the cut), which would change the kept subspace; the span of b = r + 16 of them
        // holds the exact top-r subspace to ~1e-5, and Z = A^T U0 (FP32 FMA, FP64 Gram) gives
        // the exact Ritz pairs.  The next data E_r^T Z^T replaces the projection pass.
        const int b = refine_width(st);
        npasses += 1;
        TT_TRY(launch_f64_to_f32_cols(B.evecs, m, m, b, B.yf, m, b, s));
        TT_TRY(pass.run(TT_PASS_PROJECT, 2.0 * m * cols * b, 4.0 * m * cols + 4.0 * b * cols, [&] {
          return launch_project(cur, m, cols, B.yf, b, m, B.bt, b, OUT_ROWMAJOR, 1, 1, TT_GEMM_FP32, ws, c->dstat,
                                s);
        }));
        TT_TRY(pass.run(TT_PASS_OTHER, 2.0 * cols * b * b, 4.0 * cols * b,
                        [&] { return launch_gram(B.bt, cols, b, b, 1, B.w, true, ws, s); }));
        TT_TRY(launch_syev(B.w, b, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
        k_store_sigma<<<1, 64, 0, s>>>(B.evals, std::min(b, TT_STATS_MAX_SIGMA), sigdst);
        count_launch();
        float* ubuf = B.corebuf;
        TT_TRY(launch_small_nn(B.yf, m, b, m, B.evecs, rq, b, nullptr, re, ubuf, m, s));  // U = U0 E_r
        TT_TRY(launch_canon_cols(ubuf, m, re, m, B.evecs, b, b, s));
        if (ring1) {
          TT_TRY(launch_ring_core1(ubuf, (int)m, P.r[0], P.r[1], cores[0], s));
        } else {
          TT_TRY(join_side());
          TT_TRY(emit_core(ubuf, core_dst, pend, rin, rcore, ni, rq, s));
        }
        TT_TRY(launch_f64_to_f32_cols(B.evecs, b, b, re, B.ef, b, rq, s));
        TT_TRY(pass.run(TT_PASS_OTHER, 2.0 * b * cols * nout, 4.0 * b * cols + 4.0 * nout * cols, [&] {
          return launch_project(B.bt, b, cols, B.ef, nout, b, next, st.perm231 ? 0 : nout,
                                st.perm231 ? OUT_PERM231 : OUT_ROWMAJOR, P.r[0], pr1, TT_GEMM_FP32, ws, c->dstat, s);
        }));
        pend = nullptr;
        cur = next;
        slot ^= 1;
        continue;
      }
      // basis (m x r_req, zero-padded beyond r_eff), FP32, canonical column signs
      TT_TRY(launch_f64_to_f32_cols(B.evecs, m, m, re, B.ef, m, rq, s));
      TT_TRY(launch_canon_cols(B.ef, m, re, m, B.evecs, (int)m, m, s));
      if (ring1) {
        TT_TRY(launch_ring_core1(B.ef, (int)m, P.r[0], P.r[1], cores[0], s));
      } else {
        TT_TRY(join_side());
        TT_TRY(emit_core(B.ef, core_dst, pend, rin, rcore, ni, rq, s));
      }
      if (fold) {
        if (!st.fold) --npasses;
        // next data = raw data; pending rotation = eigenvectors of the raw Gram
        double* pnew = B.pend[pend_slot ^ 1];
        TT_CUDA(cudaMemcpyAsync(pnew, B.evecs, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, s));
        pend = pnew;
        pend_slot ^= 1;
        continue;
      }
      TT_TRY(pass.run(TT_PASS_PROJECT, 2.0 * m * cols * nout, 4.0 * m * cols + 4.0 * nout * cols, [&] {
        return launch_project(cur, m, cols, B.ef, nout, m, next, st.perm231 ? 0 : nout,
                              st.perm231 ? OUT_PERM231 : OUT_ROWMAJOR, P.r[0], pr1,
                              engine, ws, c->dstat, s);
      }));
    } else if (st.path == PATH_EXACT_COLS) {
      npasses += 2;
      // W = A^T A over the rows of A (vectors = rows i, components = columns)
      TT_TRY(pass.run(TT_PASS_GRAM, 2.0 * m * cols * cols, 4.0 * m * cols,
                      [&] { return launch_gram(cur, m, (int)cols, 1, m, B.w, true, ws, s); }));
      TT_TRY(launch_syev(B.w, (int)cols, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
      k_store_sigma<<<1, 64, 0, s>>>(B.evals, (int)std::min<long long>(cols, TT_STATS_MAX_SIGMA), sigdst);
      count_launch();
      TT_TRY(decide((int)cols, 0.0));
      energy_exact = true;
      TT_TRY(launch_inv_sigma(B.evals, re, B.colscale, 1e-30, s));
      float* ubuf = B.corebuf;
      TT_TRY(pass.run(TT_PASS_OTHER, 2.0 * m * cols * rq, 4.0 * m * cols + 4.0 * m * rq, [&] {
        return launch_small_nn(cur, m, (int)cols, m, B.evecs, rq, cols, B.colscale, re, ubuf, m, s);
      }));
      TT_TRY(launch_canon_cols(ubuf, m, re, m, B.evecs, (int)cols, cols, s));
      if (ring1) {
        TT_TRY(launch_ring_core1(ubuf, (int)m, P.r[0], P.r[1], cores[0], s));
      } else {
        TT_TRY(join_side());
        TT_TRY(emit_core(ubuf, core_dst, pend, rin, rcore, ni, rq, s));
      }
      if (st.perm231) {
        float* tmp = B.bt;  // q x cols scratch (q <= 128, cols <= 128)
        TT_TRY(launch_sigma_vt(B.evals, B.evecs, (int)cols, nout, re, tmp, s));
        TT_TRY(launch_permute231(tmp, next, P.r[0], pr1, cols, s));
      } else {
        TT_TRY(launch_sigma_vt(B.evals, B.evecs, (int)cols, nout, re, next, s));
      }
    } else {  // PATH_RAND
      // One EDrSVD attempt with sketch width ksa and pwa power iterations: Q (B.yf), B^T
      // (B.bt), the eigen-decomposition of B B^T (B.evals / B.evecs), sigma stored.
      // tc_b: form B on the tensor cores even with adaptive ranks (a learned attempt judged by
      // the probe estimate, which does not read B's energy).
      auto attempt = [&](int ksa, int pwa, unsigned sid, bool tc_b) -> int {
        TT_TRY(launch_gaussian(B.omega, cols, ksa, cols, o.seed, sid, s));
        const double fl_pass = 2.0 * m * cols * ksa;
        const double by_pass = 4.0 * m * cols + 4.0 * cols * ksa;
        TT_TRY(pass.run(TT_PASS_SKETCH, fl_pass, by_pass, [&] {
          return launch_sketch(cur, m, cols, B.omega, ksa, 1, cols, B.yd, engine, ws, c->dstat, s);
        }));
        TT_TRY(launch_f64_to_f32_cols(B.yd, m, m, ksa, B.yf, m, ksa, s));
        TT_TRY(launch_cholqr2(B.yf, m, ksa, 1, m, nullptr, ws, c->dstat, s));
        for (int it = 0; it < pwa; ++it) {
          // Z = A^T Q written column-major (cols x ksa), the layout the sketch reads W in
          TT_TRY(pass.run(TT_PASS_PROJECT, fl_pass, by_pass, [&] {
            return launch_project(cur, m, cols, B.yf, ksa, m, B.bt, cols, OUT_COLMAJOR, 1, 1, engine, ws, c->dstat,
                                  s);
          }));
          // Adaptive ranks need the basis beyond the FP32 Gram's resolution (graded spectra
          // down to delta / ||A|| ~ 1e-4): the pass forms its Gram with FP64 products there.
          TT_TRY(pass.run(TT_PASS_OTHER, 4.0 * cols * ksa * ksa, 12.0 * cols * ksa, [&] {
            return launch_orth_power(B.bt, cols, ksa, 1, cols, ws, c->dstat, s, adaptive);
          }));
          TT_TRY(pass.run(TT_PASS_SKETCH, fl_pass, by_pass, [&] {
            return launch_sketch(cur, m, cols, B.bt, ksa, 1, cols, B.yd, engine, ws, c->dstat, s);
          }));
          TT_TRY(launch_f64_to_f32_cols(B.yd, m, m, ksa, B.yf, m, ksa, s));
          TT_TRY(launch_cholqr2(B.yf, m, ksa, 1, m, nullptr, ws, c->dstat, s));
        }
        // B^T = A^T Q (cols x ksa, row-major) = B (ksa x cols, column-major).  Adaptive ranks
        // take ||B||^2 as the captured energy, which must hold ~1e-8 relative.  Tensor-core
        // accumulation (FP32 in TMEM, truncating) shrinks long product-sums by ~1e-6 relative
        // even with exact 3xTF32 products, more than delta^2; that mode forms B on the FP32
        // engine (round-to-nearest FMA).
        TT_TRY(pass.run(TT_PASS_PROJECT, fl_pass, by_pass, [&] {
          return launch_project(cur, m, cols, B.yf, ksa, m, B.bt, ksa, OUT_ROWMAJOR, 1, 1,
                                (adaptive && !tc_b) ? TT_GEMM_FP32 : engine, ws, c->dstat, s);
        }));
        // Gram of the small factor B (ksa x cols, column-major = B^T row-major): the input of
        // the eigen-based small SVD (TT3O:717), on the tensor cores for long B.
        // Adaptive ranks read ||A||^2 - sum(lambda) down to delta^2 = eps^2 ||X||^2 / (d - 1): the
        // eigenvalue sum must then hold ~1e-8 relative, which the tensor-core Gram (TF32
        // operands, FP32 accumulation within 2048-column units) does not guarantee on short B.
        TT_TRY(pass.run(TT_PASS_OTHER, 2.0 * cols * ksa * ksa, 4.0 * cols * ksa, [&] {
          if (engine == TT_GEMM_TC && !adaptive) {
            const int rc = launch_gram_tc(B.bt, ksa, cols, B.w, ws, c->dstat, s);
            if (rc != TT_ERR_UNSUPPORTED) return rc;
          }
          return launch_gram(B.bt, cols, ksa, ksa, 1, B.w, true, ws, s);
        }));
        // Fixed ranks keep the first re <= 16 eigenpairs of a wide sketch's Gram: above 64 the
        // subspace solver's 32 Ritz pairs (the eigenvalues beyond them are reported as 0).
        if (!adaptive && ksa > 64 && re <= 16)
          TT_TRY(launch_syev_top(B.w, ksa, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
        else
          TT_TRY(launch_syev(B.w, ksa, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
        k_store_sigma<<<1, 64, 0, s>>>(B.evals, std::min(ksa, TT_STATS_MAX_SIGMA), sigdst);
        count_launch();
        npasses += 2 + 2 * pwa;
        ++natt;
        return TT_OK;
      };
      double step_outside = 0.0;  // energy outside the accepted attempt's subspace
      bool learned_step = false;   // accepted on the probe estimate (B and its energy from TF32 tiles)
      // Energy outside the attempt's subspace: ||A||^2 - ||B||^2, with ||A||^2 the exact carried
      // energy (recomputed by one FP64 norm pass when a learned step left an estimate).
      auto outside = [&](int ksa, double* out) -> int {
        if (!energy_exact) {
          const size_t mk = ws.mark();
          double* acc = ws.take<double>(2);
          if (!acc) {
            set_error(TT_ERR_NOMEM, "norm accumulator");
            return TT_ERR_NOMEM;
          }
          TT_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s));
          TT_TRY(launch_diff_norm(cur, nullptr, m * cols, acc, s));
          double h[2];
          TT_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
          TT_CUDA(cudaStreamSynchronize(s));
          ws.reset(mk);
          energy = h[1];
          energy_exact = true;
        }
        std::vector<double> lam((size_t)ksa);
        TT_CUDA(cudaMemcpyAsync(lam.data(), B.evals, sizeof(double) * ksa, cudaMemcpyDeviceToHost, s));
        TT_CUDA(cudaStreamSynchronize(s));
        double kept = 0.0;
        for (double v : lam) kept += std::max(v, 0.0);
        *out = energy - kept;
        step_outside = *out;
        return TT_OK;
      };
      const int ks_cap = st.ks;
      int ks = ks_cap, pw = o.power_iters;
      const bool adapt_ks = adaptive && (o.flags & (TT_FLAG_ADAPTIVE_KS | TT_FLAG_LEARNED));
      if (!adapt_ks) {
        TT_TRY(attempt(ks, pw, (unsigned)k, false));
        if (adaptive) {
          double out = 0.0;
          TT_TRY(outside(ks, &out));
        }
      } else {
        bool done = false;
        int ks_next = std::min(ks_cap, 16 + std::max(0, o.oversample));
        unsigned sid = (unsigned)k;
        if ((o.flags & TT_FLAG_LEARNED) && ks_cap >= TT_PROBE_COLS) {
          if (!c->pred) {
            set_error(TT_ERR_ARG, "TT_FLAG_LEARNED without a predictor (tt_ctx_set_predictor)");
            return TT_ERR_ARG;
          }
          // probe: Y0 = A Omega0 (TT_PROBE_COLS columns) on the FP32 engine (exact products, FP64
          // sums), eigenvalues of Y0^T Y0, features.  Y0 is kept: it also measures the energy the
          // attempt leaves outside its subspace (the a-posteriori estimate below).
          float* feat = c->pred + TT_MLP_PARAMS;
          float* yout = feat + TT_MLP_INPUTS;
          TT_TRY(launch_gaussian(B.omega, cols, TT_PROBE_COLS, cols, o.seed, 0x40000000u + (unsigned)k, s));
          TT_TRY(pass.run(TT_PASS_SKETCH, 2.0 * m * cols * TT_PROBE_COLS, 4.0 * m * cols + 4.0 * cols * TT_PROBE_COLS,
                          [&] {
                            return launch_sketch(cur, m, cols, B.omega, TT_PROBE_COLS, 1, cols, B.y0, TT_GEMM_FP32,
                                                 ws, c->dstat, s);
                          }));
          ++npasses;
          TT_TRY(launch_f64_to_f32_cols(B.y0, m, m, TT_PROBE_COLS, B.yf, m, TT_PROBE_COLS, s));
          TT_TRY(launch_gram(B.yf, m, TT_PROBE_COLS, 1, m, B.w, true, ws, s));
          TT_TRY(launch_syev(B.w, TT_PROBE_COLS, B.evals, B.evecs, max_sweeps, ws, c->dstat, s));
          const double tol = energy > 0.0 ? std::sqrt(delta2 / energy) : 1.0;
          TT_TRY(launch_probe_features(B.evals, energy, tol, m, cols, feat, s));
          TT_TRY(launch_mlp_forward(c->pred, feat, 1, yout, s));
          float hy[TT_MLP_OUTPUTS];
          TT_CUDA(cudaMemcpyAsync(hy, yout, sizeof(hy), cudaMemcpyDeviceToHost, s));
          TT_CUDA(cudaStreamSynchronize(s));
          // decode: rank 2^(10 y0), oversampling 2^(5 y1), power iterations 2 y2
          const double rh = std::max(1.0, std::round(std::exp2(std::min(10.0 * (double)hy[0], 10.0))));
          const int sh = (int)std::lround(std::exp2(std::min(std::max(5.0 * (double)hy[1], 1.0), 5.0)));
          pw = (int)std::lround(std::min(std::max(2.0 * (double)hy[2], 0.0), 3.0));
          ks = (int)std::min<double>((double)ks_cap, std::max(1.0, rh + sh));
          if (10 * ks >= 9 * ks_cap) ks = ks_cap;  // within 10 % of the width limit: use the limit
          // B on the tensor cores unless their rounding noise in B (TF32 operands: relative RMS
          // ~2e-4 per element, of which the fraction ks/m lands in B) could reach 5 % of the budget.
          const bool tc_b = engine == TT_GEMM_TC && (double)ks / (double)m * 4e-8 * energy <= 0.05 * delta2;
          TT_TRY(attempt(ks, pw, sid, tc_b));
          // A-posteriori estimate of the energy outside range(Q) (Halko, Martinsson & Tropp 2011,
          // sec. 4.3): for Gaussian omega, E||(I - QQ^T) A omega||^2 = ||(I - QQ^T) A||_F^2, so the
          // mean over the probe columns is unbiased; two standard errors of the mean are added.
          TT_TRY(launch_probe_resid(B.yf, m, ks, m, B.y0, m, TT_PROBE_COLS, B.resid, s));
          double hr[TT_PROBE_COLS];
          lam_pre.assign((size_t)ks, 0.0);
          TT_CUDA(cudaMemcpyAsync(hr, B.resid, sizeof(hr), cudaMemcpyDeviceToHost, s));
          TT_CUDA(cudaMemcpyAsync(lam_pre.data(), B.evals, sizeof(double) * ks, cudaMemcpyDeviceToHost, s));
          TT_CUDA(cudaStreamSynchronize(s));
          double mean = 0.0, var = 0.0;
          for (double v : hr) mean += v;
          mean /= TT_PROBE_COLS;
          for (double v : hr) var += (v - mean) * (v - mean);
          var /= (TT_PROBE_COLS - 1);
          const double est = mean + 2.0 * std::sqrt(var / TT_PROBE_COLS);
          if (est <= delta2 || ks >= ks_cap) {
            done = true;
            step_outside = est;
            learned_step = tc_b;
          } else {
            ++nfall;
            lam_pre.clear();
            ks_next = std::min(ks_cap, std::max(2 * ks, ks_next));
            pw = o.power_iters;
          }
        }
        while (!done) {
          ks = ks_next;
          pw = o.power_iters;
          TT_TRY(attempt(ks, pw, sid + 0x1000u * (unsigned)natt, false));
          double out = 0.0;
          TT_TRY(outside(ks, &out));
          if (out <= delta2 || ks >= ks_cap) done = true;
          ks_next = std::min(ks_cap, 2 * ks);
        }
      }
      step_ks[k] = ks;
      step_pw[k] = pw;
      step_att[k] = natt - natt0;
      TT_TRY(decide(ks, step_outside));
      energy_exact = !learned_step;
      // core = Q E_r with canonical column signs (E's columns follow)
      float* ubuf = B.corebuf;
      TT_TRY(launch_small_nn(B.yf, m, ks, m, B.evecs, rq, ks, nullptr, re, ubuf, m, s));
      TT_TRY(launch_canon_cols(ubuf, m, re, m, B.evecs, ks, ks, s));
      // next = E_r^T B  (rotation of the small factor; plain FP32 keeps it exact to FP32)
      TT_TRY(launch_f64_to_f32_cols(B.evecs, ks, ks, re, B.ef, ks, rq, s));
      TT_TRY(pass.run(TT_PASS_OTHER, 2.0 * ks * cols * nout, 4.0 * ks * cols + 4.0 * nout * cols, [&] {
        return launch_project(B.bt, ks, cols, B.ef, nout, ks, next, st.perm231 ? 0 : nout,
                              st.perm231 ? OUT_PERM231 : OUT_ROWMAJOR, P.r[0], pr1, TT_GEMM_FP32,
                              ws, c->dstat, s);
      }));
      if (ring1) {
        TT_TRY(launch_ring_core1(ubuf, (int)m, P.r[0], P.r[1], cores[0], s));
      } else {
        TT_TRY(join_side());
        TT_TRY(emit_core(ubuf, core_dst, pend, rin, rcore, ni, rq, s));
      }
    }
    pend = nullptr;
    cur = next;
    slot ^= 1;
  }
  // last core: (r_{d-1}, n_d, r_d) from the current data (P.last_rows rows per index), with a
  // pending rotation folded in or compacted rows restored as zeros
  {
    const int k = P.d - 1;
    const long long ni = P.n[k] * (long long)P.r[P.d];
    TT_TRY(join_side());
    TT_TRY(emit_core(cur, cores[k], pend, P.last_rows, P.r[k], ni, 1, s));
  }
  TT_TRY(join_side());
  TT_CUDA(cudaEventRecord(c->ev1, s));
  if (host_io) {
    for (int k = 0; k < P.d; ++k)
      TT_CUDA(cudaMemcpyAsync(cores_out[k], cores[k], sizeof(float) * core_elems(P, k),
                              cudaMemcpyDeviceToHost, s));
  }
  TT_CUDA(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
  TT_CUDA(cudaMemcpyAsync(c->hsig, c->dsig, sizeof(double) * TT_MAX_ORDER * TT_STATS_MAX_SIGMA,
                          cudaMemcpyDeviceToHost, s));
  TT_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    stats->ms = ms;
    stats->nsteps = nsteps;
    for (int k = 0; k <= P.d; ++k) stats->ranks[k] = P.r[k];
    stats->est_rel_err = adaptive && xnorm2 > 0.0 ? std::sqrt(tail_sum / xnorm2) : 0.0;
    stats->passes = npasses;
    stats->fallbacks = nfall;
    stats->eps_unmet = eps_unmet;
    for (int k = 0; k < nsteps && k < TT_MAX_ORDER; ++k) {
      stats->step_ks[k] = step_ks[(size_t)k];
      stats->step_power[k] = step_pw[(size_t)k];
      stats->step_attempts[k] = step_att[(size_t)k];
    }
    for (int k = 0; k < nsteps; ++k) {
      int cnt = 0;
      for (int i = 0; i < TT_STATS_MAX_SIGMA; ++i) {
        const double v = c->hsig[(size_t)k * TT_STATS_MAX_SIGMA + i];
        if (v < 0) break;
        stats->sigma[k][i] = (float)v;
        ++cnt;
      }
      stats->nsigma[k] = cnt;
    }
    stats->jacobi_sweeps = c->hstat->sweeps;
    stats->kernels = g_kernel_launches;
    stats->flops = pass.flops;
    stats->bytes = pass.bytes;
    stats->top_kind = -1;
    stats->top_step = -1;
    for (const PassRec& rec : pass.recs) {
      float pm = 0.f;
      cudaEventElapsedTime(&pm, rec.a, rec.b);
      stats->pass_ms[rec.kind] += pm;
      stats->pass_bytes[rec.kind] += rec.bytes;
      stats->pass_launches[rec.kind] += 1;
      if (pm > stats->top_ms) {
        stats->top_ms = pm;
        stats->top_kind = rec.kind;
        stats->top_step = rec.step;
        stats->top_bytes = rec.bytes;
      }
    }
  }
  if (c->hstat->code != 0) {
    set_error(c->hstat->code, "device status %d (detail %d)", c->hstat->code, c->hstat->detail);
    return c->hstat->code;
  }
  if (eps_unmet > 0 && (o.flags & TT_FLAG_STRICT_EPS)) {
    set_error(TT_ERR_RANK, "eps = %g not met: %d unfolding(s) reached their rank bound with more than delta^2 "
              "discarded (est. rel. error %.3e)", o.eps, eps_unmet,
              xnorm2 > 0.0 ? std::sqrt(tail_sum / xnorm2) : 0.0);
    return TT_ERR_RANK;
  }
  return TT_OK;
}

int run_entry(tt_ctx* c, const float* x, int d, const int* n, const int* r, const tt_opts* opts,
              float* const* cores, tt_stats* stats, bool ring) {
  if (!c || !x || !cores) {
    set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  tt_opts o;
  if (opts)
    o = *opts;
  else
    tt_default_opts(&o);
  if (o.eps < 0.0 || o.eps != o.eps) {
    set_error(TT_ERR_ARG, "eps must be >= 0");
    return TT_ERR_ARG;
  }
  if ((o.flags & (TT_FLAG_ADAPTIVE_KS | TT_FLAG_LEARNED)) && !(o.eps > 0.0)) {
    set_error(TT_ERR_ARG, "TT_FLAG_ADAPTIVE_KS / TT_FLAG_LEARNED need eps > 0");
    return TT_ERR_ARG;
  }
  if ((o.flags & TT_FLAG_LEARNED) && !c->pred) {
    set_error(TT_ERR_ARG, "TT_FLAG_LEARNED without a predictor (tt_ctx_set_predictor)");
    return TT_ERR_ARG;
  }
  if (o.flags & TT_FLAG_HOST_STREAM) {
    if (ring || o.eps > 0.0 || (o.flags & (TT_FLAG_CHECK_FINITE | TT_FLAG_ADAPTIVE_KS | TT_FLAG_LEARNED))) {
      set_error(TT_ERR_UNSUPPORTED, "TT_FLAG_HOST_STREAM: TT-SVD with fixed ranks only");
      return TT_ERR_UNSUPPORTED;
    }
    o.flags |= TT_FLAG_NO_FOLD;  // the first projection is materialised from the streamed chunks
    o.flags &= ~TT_FLAG_IDENTITY_GAUGE;
  }
  if (o.eps > 0.0) {
    if (ring) {
      set_error(TT_ERR_UNSUPPORTED, "adaptive ranks (eps > 0) are implemented for TT-SVD only");
      return TT_ERR_UNSUPPORTED;
    }
    // The rank of a full-rank step is not known in advance: no step is planned as a fold, and
    // run_chain folds a step whose chosen rank keeps every row unless the caller said no.
    if (!(o.flags & TT_FLAG_NO_FOLD)) o.flags |= kFlagAdaptiveFold;
    o.flags |= TT_FLAG_NO_FOLD;
  }
  Plan P;
  TT_TRY(make_plan(d, n, r, ring, o, P));
  if (o.flags & TT_FLAG_HOST_STREAM) {
    const Step& s0 = P.steps[0];
    if (s0.path != PATH_EXACT_ROWS) {
      set_error(TT_ERR_UNSUPPORTED, "TT_FLAG_HOST_STREAM needs a first unfolding with <= %d rows (got %lld x %lld)",
                TT_MAX_SMALL, s0.m, s0.cols);
      return TT_ERR_UNSUPPORTED;
    }
    P.stream_cols = std::max<long long>(1, std::min<long long>(s0.cols, (long long)(c->chunk_bytes / (4 * s0.m))));
    // the Gram and projection kernels see one chunk at a time
    P.max_ws = std::max(P.max_ws, gram_ws_bytes(P.stream_cols, (int)s0.m));
    P.max_ws = std::max(P.max_ws, gram_tc_ws_bytes(s0.m, P.stream_cols));
    P.max_ws = std::max(P.max_ws, gram32x_ws_bytes());
    P.max_ws = std::max(P.max_ws, project_ws_bytes(s0.m, P.stream_cols, s0.r_req));
  }
  for (int k = 0; k < d; ++k)
    if (!cores[k]) {
      set_error(TT_ERR_ARG, "null core pointer %d", k);
      return TT_ERR_ARG;
    }
  return run_chain(c, x, P, o, cores, stats);
}

}  // namespace

extern "C" int tt_svd(tt_ctx* ctx, const float* x, int d, const int* n, const int* r,
                      const tt_opts* opts, float* const* cores, tt_stats* stats) {
  return run_entry(ctx, x, d, n, r, opts, cores, stats, false);
}

extern "C" int tr_svd(tt_ctx* ctx, const float* x, int d, const int* n, const int* r,
                      const tt_opts* opts, float* const* cores, tt_stats* stats) {
  return run_entry(ctx, x, d, n, r, opts, cores, stats, true);
}

extern "C" int tt_rel_error(tt_ctx* c, const float* x, int d, const int* n, const int* r, int ring,
                            const float* const* cores, double* rel_err) {
  if (!c || !x || !n || !r || !cores || !rel_err) {
    set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  if (d < 2 || d > TT_MAX_ORDER) {
    set_error(TT_ERR_SHAPE, "order %d", d);
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  long long N = 1;
  for (int k = 1; k < d; ++k) N *= n[k];
  // merged right part M_k sizes: r_{k-1} * (n_k ... n_d) * r_d
  // M_k (cores k..d-1 merged) holds r[k] * n[k] * ... * n[d-1] * r[d] floats.
  long long maxm = 0;
  {
    long long rest = r[d];
    for (int k = d - 1; k >= 1; --k) {
      rest *= n[k];
      maxm = std::max(maxm, (long long)r[k] * rest);
    }
  }
  TT_TRY(tt_ctx_reserve(c, sizeof(float) * (size_t)maxm * 2 + 4096 + (1 << 20)));
  Arena a{c->arena, c->cap, 0};
  float* buf[2] = {a.take<float>(maxm), a.take<float>(maxm)};
  double* acc = a.take<double>(2);
  if (!buf[1] || !acc) {
    set_error(TT_ERR_NOMEM, "error workspace");
    return TT_ERR_NOMEM;
  }
  cudaStream_t s = c->stream;
  const float* mk = cores[d - 1];
  long long cols = (long long)n[d - 1] * r[d];
  int sl = 0;
  for (int k = d - 2; k >= 1; --k) {
    // M_k = G_k (r_{k-1} n_k x r_k) * M_{k+1} (r_k x cols)
    TT_TRY(launch_gemm_nn(cores[k], (long long)r[k] * n[k], r[k + 1], mk, cols, buf[sl], s));
    mk = buf[sl];
    sl ^= 1;
    cols *= n[k];
  }
  TT_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s));
  TT_TRY(launch_recon_err(x, n[0], N, cores[0], ring ? r[0] : 1, r[1], mk, acc, s));
  double h[2] = {0, 0};
  TT_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
  TT_CUDA(cudaStreamSynchronize(s));
  *rel_err = h[1] > 0 ? sqrt(h[0] / h[1]) : 0.0;
  return TT_OK;
}

// ---- building blocks ----
namespace {
int ws_for(tt_ctx* c, size_t bytes, Arena& ws) {
  TT_TRY(tt_ctx_reserve(c, bytes + (1 << 20)));
  ws = Arena{c->arena, c->cap, 0};
  return TT_OK;
}
}  // namespace

// Context accessors for the other translation units (batched path).
namespace ttr {
int ctx_arena(tt_ctx* c, size_t bytes, Arena* ws) {
  TT_CUDA(cudaSetDevice(c->device));
  return ws_for(c, bytes, *ws);
}
cudaStream_t ctx_stream(tt_ctx* c) { return c->stream; }
DevStatus* ctx_status(tt_ctx* c) { return c->dstat; }
}  // namespace ttr

namespace {
int check_status(tt_ctx* c) {
  TT_CUDA(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
  TT_CUDA(cudaStreamSynchronize(c->stream));
  if (c->hstat->code) {
    set_error(c->hstat->code, "device status %d (detail %d)", c->hstat->code, c->hstat->detail);
    return c->hstat->code;
  }
  return TT_OK;
}
}  // namespace

#define TT_NEED(p)                                \
  do {                                            \
    if (!(p)) {                                   \
      set_error(TT_ERR_ARG, "null argument " #p); \
      return TT_ERR_ARG;                          \
    }                                             \
  } while (0)

extern "C" int tt_ctx_set_wait_limit(tt_ctx* c, unsigned long long ns) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  TT_CUDA(cudaSetDevice(c->device));
  return set_wait_limit_ns(ns);
}

extern "C" int tt_k_wait_selftest(tt_ctx* c) {
  if (!c) {
    set_error(TT_ERR_ARG, "null ctx");
    return TT_ERR_ARG;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  TT_TRY(launch_wait_selftest(c->dstat, c->stream));
  return check_status(c);
}

extern "C" int tt_k_gaussian(tt_ctx* c, float* out, long long rows, int cols, long long ld,
                             unsigned long long seed, unsigned stream_id) {
  TT_NEED(c);
  TT_NEED(out);
  if (rows < 0 || cols < 0 || ld < rows) {
    set_error(TT_ERR_SHAPE, "gaussian shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_gaussian(out, rows, cols, ld, seed, stream_id, c->stream));
  TT_CUDA(cudaStreamSynchronize(c->stream));
  return TT_OK;
}

extern "C" int tt_k_sketch(tt_ctx* c, const float* a, long long m, long long n, const float* w,
                           int N, long long ldw, double* y, int gemm) {
  TT_NEED(c);
  TT_NEED(a);
  TT_NEED(w);
  TT_NEED(y);
  if (gemm < TT_GEMM_AUTO || gemm > TT_GEMM_FP32) {
    set_error(TT_ERR_ARG, "gemm option %d (expected TT_GEMM_AUTO, TT_GEMM_TC or TT_GEMM_FP32)", gemm);
    return TT_ERR_ARG;
  }
  if (m < 1 || n < 1 || N < 1 || ldw < n) {
    set_error(TT_ERR_SHAPE, "sketch shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, sketch_ws_bytes(m, n, N) * 2, ws));
  const int eng = (gemm == TT_GEMM_FP32 || !tc_available()) ? TT_GEMM_FP32 : TT_GEMM_TC;
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  TT_TRY(launch_sketch(a, m, n, w, N, 1, ldw, y, eng, ws, c->dstat, c->stream));
  return check_status(c);
}

extern "C" int tt_k_gaussian_rows(tt_ctx* c, float* out, long long row0, long long nrows, long long total_rows,
                                  int cols, long long ld, unsigned long long seed, unsigned stream_id) {
  TT_NEED(c);
  TT_NEED(out);
  if (row0 < 0 || nrows < 0 || row0 + nrows > total_rows || cols < 0 || ld < nrows) {
    set_error(TT_ERR_SHAPE, "gaussian_rows shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_gaussian_rows(out, row0, nrows, total_rows, cols, ld, seed, stream_id, c->stream));
  return TT_OK;
}

extern "C" int tt_probe_features(tt_ctx* c, const float* a, long long m, long long n, double energy, double tol,
                                 unsigned long long seed, unsigned stream_id, float* features) {
  TT_NEED(c);
  TT_NEED(a);
  TT_NEED(features);
  if (m < 1 || n < 1) {
    set_error(TT_ERR_SHAPE, "probe_features shape %lld x %lld", m, n);
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  const int P = TT_PROBE_COLS;
  tt_opts o;
  tt_default_opts(&o);
  const int engine = engine_for(o, m, n);
  const size_t bytes = sizeof(float) * (size_t)n * P + sizeof(double) * (size_t)m * P + sizeof(float) * (size_t)m * P +
                       sizeof(double) * (2 * P * P + P + 2) + sketch_ws_bytes(m, n, P) + gram_ws_bytes(m, P) +
                       (size_t)TT_MAX_SMALL * TT_MAX_SMALL * sizeof(double) * 8 + 16 * 4096;
  Arena ws;
  TT_TRY(ws_for(c, bytes, ws));
  float* om = ws.take<float>((size_t)n * P);
  double* yd = ws.take<double>((size_t)m * P);
  float* yf = ws.take<float>((size_t)m * P);
  double* w = ws.take<double>((size_t)P * P);
  double* ev = ws.take<double>((size_t)P);
  double* vec = ws.take<double>((size_t)P * P);
  double* acc = ws.take<double>(2);
  if (!om || !yd || !yf || !w || !ev || !vec || !acc) {
    set_error(TT_ERR_NOMEM, "probe workspace");
    return TT_ERR_NOMEM;
  }
  cudaStream_t s = c->stream;
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), s));
  if (energy < 0.0) {
    TT_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s));
    TT_TRY(launch_diff_norm(a, nullptr, m * n, acc, s));
    double h[2];
    TT_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
    TT_CUDA(cudaStreamSynchronize(s));
    energy = h[1];
  }
  TT_TRY(launch_gaussian(om, n, P, n, seed, stream_id, s));
  TT_TRY(launch_sketch(a, m, n, om, P, 1, n, yd, engine, ws, c->dstat, s));
  TT_TRY(launch_f64_to_f32_cols(yd, m, m, P, yf, m, P, s));
  TT_TRY(launch_gram(yf, m, P, 1, m, w, true, ws, s));
  TT_TRY(launch_syev(w, P, ev, vec, 40, ws, c->dstat, s));
  TT_TRY(launch_probe_features(ev, energy, tol, m, n, features, s));
  return check_status(c);
}

extern "C" int tt_mlp_forward(tt_ctx* c, const float* params, const float* x, int n, float* y) {
  TT_NEED(c);
  TT_NEED(params);
  TT_NEED(x);
  TT_NEED(y);
  if (n < 0) {
    set_error(TT_ERR_SHAPE, "mlp_forward n = %d", n);
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_mlp_forward(params, x, n, y, c->stream));
  return TT_OK;
}

extern "C" int tt_mlp_grad(tt_ctx* c, const float* params, const float* x, const float* t, int n, float* grad,
                           float* loss) {
  TT_NEED(c);
  TT_NEED(params);
  TT_NEED(x);
  TT_NEED(t);
  TT_NEED(grad);
  if (n < 1) {
    set_error(TT_ERR_SHAPE, "mlp_grad n = %d", n);
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_mlp_train(const_cast<float*>(params), nullptr, nullptr, x, t, n, 1, n, 0.f, 0, 0ull, loss, grad, 1,
                          c->stream));
  return TT_OK;
}

extern "C" int tt_mlp_train(tt_ctx* c, float* params, float* adam_m, float* adam_v, const float* x, const float* t,
                            int n, int steps, int batch, float lr, int step0, unsigned long long seed,
                            float* loss_trace) {
  TT_NEED(c);
  TT_NEED(params);
  TT_NEED(adam_m);
  TT_NEED(adam_v);
  TT_NEED(x);
  TT_NEED(t);
  if (n < 1 || steps < 0 || batch < 1 || step0 < 0 || !(lr >= 0.f)) {
    set_error(TT_ERR_ARG, "mlp_train n %d steps %d batch %d step0 %d lr %g", n, steps, batch, step0, (double)lr);
    return TT_ERR_ARG;
  }
  if (steps == 0) return TT_OK;
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_mlp_train(params, adam_m, adam_v, x, t, n, steps, batch, lr, step0, seed, loss_trace, nullptr, 0,
                          c->stream));
  return TT_OK;
}

extern "C" int tt_k_project(tt_ctx* c, const float* a, long long m, long long n, const float* q,
                            int N, long long ldq, float* out, long long ldo, int gemm) {
  TT_NEED(c);
  TT_NEED(a);
  TT_NEED(q);
  TT_NEED(out);
  if (m < 1 || n < 1 || N < 1 || ldq < m || ldo < N) {
    set_error(TT_ERR_SHAPE, "project shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, std::max<size_t>(1 << 20, project_ws_bytes(m, n, N)), ws));
  const int eng = (gemm == TT_GEMM_FP32 || !tc_available()) ? TT_GEMM_FP32 : TT_GEMM_TC;
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  TT_TRY(launch_project(a, m, n, q, N, ldq, out, ldo, OUT_ROWMAJOR, 1, 1, eng, ws, c->dstat, c->stream));
  return check_status(c);
}

extern "C" int tt_k_gram_rows(tt_ctx* c, const float* a, long long m, long long n, double* w,
                              int gemm) {
  TT_NEED(c);
  TT_NEED(a);
  TT_NEED(w);
  if (m < 1 || n < 1 || m > TT_MAX_SMALL) {
    set_error(TT_ERR_SHAPE, "gram_rows shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, std::max(std::max(gram_ws_bytes(n, (int)m), gram_tc_ws_bytes(m, n)), gram32x_ws_bytes()), ws));
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  int rc = TT_ERR_UNSUPPORTED;
  // up to 32 rows, AUTO and FP32 take the exact CUDA-core kernel; TC forces the tensor cores
  if (gemm != TT_GEMM_TC && m <= 32) rc = launch_gram32x(a, n, (int)m, w, ws, c->dstat, c->stream);
  if (rc == TT_ERR_UNSUPPORTED && gemm != TT_GEMM_FP32 && tc_available())
    rc = launch_gram_tc(a, m, n, w, ws, c->dstat, c->stream);
  if (rc == TT_ERR_UNSUPPORTED) rc = launch_gram(a, n, (int)m, m, 1, w, false, ws, c->stream);
  TT_TRY(rc);
  return check_status(c);
}

extern "C" int tt_k_gram_tall(tt_ctx* c, const float* z, long long n, int N, long long rs,
                              long long cs, double* w) {
  TT_NEED(c);
  TT_NEED(z);
  TT_NEED(w);
  if (n < 1 || N < 1 || N > TT_MAX_SMALL) {
    set_error(TT_ERR_SHAPE, "gram_tall shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, gram_ws_bytes(n, N), ws));
  TT_TRY(launch_gram(z, n, N, rs, cs, w, true, ws, c->stream));
  TT_CUDA(cudaStreamSynchronize(c->stream));
  return TT_OK;
}

extern "C" int tt_k_cholqr2(tt_ctx* c, float* y, long long n, int N, long long ld, double* r) {
  TT_NEED(c);
  TT_NEED(y);
  if (n < 1 || N < 1 || N > TT_MAX_SMALL || ld < n) {
    set_error(TT_ERR_SHAPE, "cholqr2 shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, gram_ws_bytes(n, N) + 8 * TT_MAX_SMALL * TT_MAX_SMALL * sizeof(double), ws));
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  TT_TRY(launch_cholqr2(y, n, N, 1, ld, r, ws, c->dstat, c->stream));
  return check_status(c);
}

extern "C" int tt_k_syev(tt_ctx* c, const double* w, int N, double* evals, double* evecs,
                         int* sweeps) {
  TT_NEED(c);
  TT_NEED(w);
  TT_NEED(evals);
  TT_NEED(evecs);
  if (N < 1 || N > TT_MAX_SMALL) {
    set_error(TT_ERR_SHAPE, "syev size %d", N);
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  Arena ws;
  TT_TRY(ws_for(c, 2 * TT_MAX_SMALL * TT_MAX_SMALL * sizeof(double) + syev_ws_bytes(N, 40), ws));
  TT_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(DevStatus), c->stream));
  TT_TRY(launch_syev(w, N, evals, evecs, 40, ws, c->dstat, c->stream));
  int st = check_status(c);
  if (sweeps) *sweeps = c->hstat->sweeps;
  return st;
}

extern "C" int tt_k_permute231(tt_ctx* c, const float* in, float* out, int r0, int r1, long long n) {
  TT_NEED(c);
  TT_NEED(in);
  TT_NEED(out);
  if (r0 < 1 || r1 < 1 || n < 1 || r0 * r1 > 8192) {
    set_error(TT_ERR_SHAPE, "permute231 shape");
    return TT_ERR_SHAPE;
  }
  TT_CUDA(cudaSetDevice(c->device));
  TT_TRY(launch_permute231(in, out, r0, r1, n, c->stream));
  TT_CUDA(cudaStreamSynchronize(c->stream));
  return TT_OK;
}
