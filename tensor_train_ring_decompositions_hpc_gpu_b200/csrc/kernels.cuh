// Launchers of the TT/TR-SVD kernels.  All take device pointers and run on `stream`.
#pragma once
#include "common.cuh"

namespace ttr {

// Workspace bump allocator over one device arena.
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
  size_t mark() const { return off; }
  void reset(size_t m) { off = m; }
};

// Bytes a launcher needs from the arena (callers reserve before launching).
size_t sketch_ws_bytes(long long m, long long n, int N);
size_t gram_ws_bytes(long long nvec, int M);
size_t project_ws_bytes(long long m, long long n, int N);

// Philox Gaussian fill (column-major rows x cols, ld).
int launch_gaussian(float* out, long long rows, int cols, long long ld, unsigned long long seed,
                    unsigned stream_id, cudaStream_t s);
// Rows [row0, row0 + nrows) of the (total_rows x cols) matrix launch_gaussian would produce.
int launch_gaussian_rows(float* out, long long row0, long long nrows, long long total_rows, int cols, long long ld,
                         unsigned long long seed, unsigned stream_id, cudaStream_t s);

// Y (m x N, FP64, ld = m) = A (m x n, lda = m) * W, W element (j, c) at w[j*wj + c*wc].
// engine: TT_GEMM_FP32 or TT_GEMM_TC.
int launch_sketch(const float* a, long long m, long long n, const float* w, int N, long long wj,
                  long long wc, double* y, int engine, Arena& ws, DevStatus* st, cudaStream_t s);

// y[idx] = sum over splits of part[split * count + idx] (FP64, fixed order).
int launch_reduce_splits(const double* part, long long count, int nsplit, double* y, cudaStream_t s);

// Output modes of the projection.
enum { OUT_ROWMAJOR = 0, OUT_PERM231 = 1, OUT_COLMAJOR = 2 };

// out = A^T Q: A (m x n, lda = m), Q (m x N, ldq).  OUT_ROWMAJOR: out[j*ldo + c];
// OUT_PERM231: column c = a + r0*b of Q^T A goes to out[b + r1*(j + n*a)] (TR bond permute).
// OUT_COLMAJOR: out[j + ldo*c] (A^T Q as a column-major n x N matrix).
int launch_project(const float* a, long long m, long long n, const float* q, int N, long long ldq,
                   float* out, long long ldo, int mode, int r0, int r1, int engine, Arena& ws,
                   DevStatus* st, cudaStream_t s);

// W (M x M, FP64, ld = M) = sum_j x_j x_j^T with x_j[c] = x[j*vs + c*es], M <= 128.
// acc64: FP64 products and accumulation; else FP32 products with FP64 flush every 1024 vectors.
int launch_gram(const float* x, long long nvec, int M, long long vs, long long es, double* w,
                bool acc64, Arena& ws, cudaStream_t s);

// CholeskyQR2 on a tall FP32 matrix, element (j, c) at y[j*vs + c*es], n x N.
// Writes R (N x N, FP64, upper) when r != nullptr.
int launch_cholqr2(float* y, long long n, int N, long long vs, long long es, double* r,
                   Arena& ws, DevStatus* st, cudaStream_t s);
// One CholeskyQR pass (between power iterations): FP32-accumulated Gram, or FP64 products with
// acc64 (graded spectra, whose small directions lie below the FP32 Gram's resolution).
int launch_orth_power(float* y, long long n, int N, long long vs, long long es, Arena& ws, DevStatus* st,
                      cudaStream_t s, bool acc64 = false);

// Arena bytes launch_syev takes for N > 64 (the rotation log); 0 for N <= 64.
size_t syev_ws_bytes(int N, int max_sweeps);
// Symmetric eigen-decomposition by parallel cyclic Jacobi (FP64, N <= 128), eigenvalues descending.
int launch_syev(const double* w, int N, double* evals, double* evecs, int max_sweeps,
                Arena& ws, DevStatus* st, cudaStream_t s);
// Leading eigenpairs for 64 < N <= 128 when at most the first 16 are used: the kSubDim = 32
// Ritz pairs of a subspace iteration (columns and eigenvalues beyond them zero); other N take
// launch_syev.
int launch_syev_top(const double* w, int N, double* evals, double* evecs, int max_sweeps,
                    Arena& ws, DevStatus* st, cudaStream_t s);

// out (r0, r1, n) -> (r1, n, r0) column-major.
int launch_permute231(const float* in, float* out, int r0, int r1, long long n, cudaStream_t s);

// C (M x N, FP32, ldc) = A (M x K, FP32, lda) * B (K x N, FP64, ldb), optionally scaled
// column-wise by colscale[c] (FP64) and with columns >= nvalid set to zero.
int launch_small_nn(const float* a, long long M, int K, long long lda, const double* b, int N,
                    long long ldb, const double* colscale, int nvalid, float* c, long long ldc,
                    cudaStream_t s);

// Fold a pending row rotation into a core: out[(a + R*i) + M*b] = sum_a' P[a' + R*a] *
// in[(a' + R*i) + M*b] with M = R * ni.  In place is not allowed.
int launch_fold_rows(const float* in, float* out, const double* p, int R, long long ni, int ncols,
                     cudaStream_t s);

// Copy the first `k` columns of an FP64 (rows x ?) matrix to FP32 (rows x ncols), zero-padding.
int launch_f64_to_f32_cols(const double* in, long long rows, long long ldin, int k, float* out,
                           long long ldout, int ncols, cudaStream_t s);

// next (k x n) = diag(sqrt(evals[0:k])) * V[:, 0:k]^T, V (n x n, FP64), rows >= kvalid zeroed.
int launch_sigma_vt(const double* evals, const double* v, int n, int k, int kvalid, float* out,
                    cudaStream_t s);

// Column scale helper for U = A V / sigma: colscale[a] = 1/sigma_a (0 when sigma tiny).
int launch_inv_sigma(const double* evals, int k, double* colscale, double rel_floor, cudaStream_t s);

// Ring core 1: core[a + r0*(i + n1*b)] = u[i + n1*(a + r0*b)].
int launch_ring_core1(const float* u, int n1, int r0, int r1, float* core, cudaStream_t s);

// Column sign convention: largest-magnitude entry of each of the first r columns of U made
// positive; the same columns of the FP64 companion (K rows, ldc) are negated alongside.
int launch_canon_cols(float* u, long long m, int r, long long ldu, double* comp, int K,
                      long long ldc, cudaStream_t s);

// out[j] = ||y_j - Q Q^T y_j||^2 (FP64) for the nq columns of Y0 (m x nq, FP64, ldy);
// Q (m x ks, FP32, ldq) with orthonormal columns.
int launch_probe_resid(const float* q, long long m, int ks, long long ldq, const double* y0, long long ldy, int nq,
                       double* out, cudaStream_t s);

// NaN/Inf scan; *flag set to 1 when found.
int launch_check_finite(const float* x, long long count, int* flag, cudaStream_t s);

// Sum of squares (FP64) of (x - y) and of x, accumulated into acc[0], acc[1].
int launch_diff_norm(const float* x, const float* y, long long count, double* acc, cudaStream_t s);

// Dense C (M x N) = A (M x K) * B (K x N), all FP32 column-major, small K (core merging).
int launch_gemm_nn(const float* a, long long M, int K, const float* b, long long N, float* c,
                   cudaStream_t s);

// Fused reconstruction check of a ring/train: acc += sum_J ||X[:, J] - sum_a G1[a] M[:, J, a]||^2
// and ||X||^2, where G1 is (r0, n1, r1) and M is (r1, N, r0).
int launch_recon_err(const float* x, int n1, long long N, const float* g1, int r0, int r1,
                     const float* mrg, double* acc, cudaStream_t s);

// Learned predictor (mlp.cu).  Features from the descending probe eigenvalues mu
// (TT_PROBE_COLS of them); network inference; training (mode 0: Adam steps on Philox-drawn
// minibatches; mode 1: gradient over samples 0..batch-1 into grad_out).
int launch_probe_features(const double* mu, double energy, double tol, long long m, long long n, float* out,
                          cudaStream_t s);
int launch_mlp_forward(const float* params, const float* x, int n, float* y, cudaStream_t s);
int launch_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* t, int n, int steps,
                     int batch, float lr, int step0, unsigned long long seed, float* loss_trace, float* grad_out,
                     int mode, cudaStream_t s);

// Context accessors (driver.cu): a workspace arena of at least `bytes`, the context stream and
// its device status word.
int ctx_arena(tt_ctx* c, size_t bytes, Arena* ws);
cudaStream_t ctx_stream(tt_ctx* c);
DevStatus* ctx_status(tt_ctx* c);

// out (Rout x cols) from in (Rin x cols), rows Rin..Rout-1 zero; column-major.
int launch_expand_rows(const float* in, int Rin, float* out, int Rout, long long cols, cudaStream_t s);

// Exact Gram W (M x M, FP64, ld = M) = sum_j x_j x_j^T of nvec contiguous M-float vectors
// (M <= 32, M % 4 == 0, 16-byte aligned base) on the CUDA cores: FP32 products, FP64 sums.
// TT_ERR_UNSUPPORTED (nothing launched) when the shape or device does not fit.
size_t gram32x_ws_bytes();
int launch_gram32x(const float* x, long long nvec, int M, double* w, Arena& ws, DevStatus* st, cudaStream_t s);

// Sketch variants that take their split-K scratch from the caller (no allocation).
int launch_sketch_tc_static(const float* a, long long m, long long n, const float* w, int N,
                            long long wj, long long wc, double* y, double* part, size_t part_cap,
                            DevStatus* st, cudaStream_t s);
int launch_sketch_simt_static(const float* a, long long m, long long n, const float* w, int N,
                              long long wj, long long wc, double* y, double* part, size_t part_cap,
                              cudaStream_t s);

// Wall-clock limit (ns, 0 = default 2 s) of the pipeline waits of the TMA kernels on the
// current device, and a self-test kernel whose wait can only run out (TT_ERR_TIMEOUT).
int set_wait_limit_ns(unsigned long long ns);
int launch_wait_selftest(DevStatus* st, cudaStream_t s);

// Tensor-core engine availability (sm_100 device, TMA encoder found, TTR_DISABLE_TC unset).
bool tc_available();
size_t sketch_tc_ws_bytes(long long m, long long n, int N);
size_t gram_tc_ws_bytes(long long m, long long n);
// W (m x m, FP64, ld = m) = A A^T on the tensor cores, A column-major m x n, m <= 128.
int launch_gram_tc(const float* a, long long m, long long n, double* w, Arena& ws, DevStatus* st,
                   cudaStream_t s);
int launch_sketch_tc(const float* a, long long m, long long n, const float* w, int N, long long wj,
                     long long wc, double* y, Arena& ws, DevStatus* st, cudaStream_t s);
int launch_project_tc(const float* a, long long m, long long n, const float* q, int N,
                      long long ldq, float* out, long long ldo, int mode, int r0, int r1,
                      Arena& ws, DevStatus* st, cudaStream_t s);

}  // namespace ttr
