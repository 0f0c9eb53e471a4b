/*
 * ttrsvd.h - C ABI of the B200 (sm_100a) TT-SVD / TR-SVD library (libttrsvd.so).
 *
 * All matrices are column-major FP32 unless stated otherwise; tensors are column-major
 * with mode 1 fastest, X(i1..id) at i1 + n1*(i2 + n2*(...)), exactly as the reference's
 * GPU programs store them.  Every entry point returns a tt_status code; the message of
 * the last failure on the calling thread is available from tt_last_error().
 *
 * Reference interfaces each entry point replaces are cited as file:line relative to the
 * reference repository (YangletLiu/Tensor_Train_Ring_Decompositions_HPC_GPU).
 */
#ifndef TTRSVD_H
#define TTRSVD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TTRSVD_ABI_VERSION 4
#define TT_MAX_ORDER 16
#define TT_MAX_SMALL 128 /* largest Gram / Jacobi size handled on chip */
#define TT_MLP_INPUTS 8    /* probe features per unfolding (tt_probe_features) */
#define TT_MLP_OUTPUTS 3   /* predicted log2 rank / 10, log2 oversampling / 5, power iterations / 2 */
#define TT_MLP_PARAMS 4931 /* 8 -> 64 -> 64 -> 3 ReLU network, packed W1 b1 W2 b2 W3 b3 */
#define TT_PROBE_COLS 16   /* Gaussian probe columns behind the features */
#define TT_LEARNED_MAX_S 32 /* largest oversampling the learned predictor may choose */

/* Status codes.  The reference aborts through assert() on every library status
 * (e.g. ttdecomposition/high_order_GPUs/ttdec6_singleGPU.cu:826-831); here every failure
 * is a return code. */
typedef enum tt_status {
  TT_OK = 0,
  TT_ERR_ARG = 1,        /* null pointer, bad flag or option */
  TT_ERR_SHAPE = 2,      /* order, mode sizes or leading dimensions invalid */
  TT_ERR_RANK = 3,       /* ranks invalid (r0 != rd for a ring, rank < 1, ...) */
  TT_ERR_NONFINITE = 4,  /* NaN or Inf found in the input (TT_FLAG_CHECK_FINITE) */
  TT_ERR_NOMEM = 5,      /* device or pinned allocation failed */
  TT_ERR_NOCONV = 6,     /* Jacobi eigen-solver did not converge within max_sweeps */
  TT_ERR_TIMEOUT = 7,    /* a bounded device-side wait ran out */
  TT_ERR_CUDA = 8,       /* CUDA runtime error */
  TT_ERR_UNSUPPORTED = 9, /* shape/rank combination outside the implemented range */
  TT_ERR_IO = 10          /* core file missing, unreadable, truncated or not a core file */
} tt_status;

/* GEMM engine for the two bulk GEMMs (sketch Y = A*W and projection B^T = A^T*Q). */
enum {
  TT_GEMM_AUTO = 0, /* tensor cores where the shape allows it */
  TT_GEMM_TC = 1,   /* tcgen05 TF32 tensor-core tiles fed by TMA, FP32 accumulation in TMEM */
  TT_GEMM_FP32 = 2  /* plain FP32 FMA (CUDA cores): the "plain FP32" form */
};

/* Per-unfolding factorisation. */
enum {
  TT_METHOD_EDRSVD = 0, /* randomized range finder + small eigen-SVD (basicRandSVD_LU) */
  TT_METHOD_EXACT = 1   /* exact Gram-eigen step (longMatrixSVD_Eign_once_device); min(m,n) <= TT_MAX_SMALL */
};

/* Option flags. */
enum {
  TT_FLAG_HOST_IO = 1,        /* x and the cores are host pointers (copied in/out inside the call) */
  TT_FLAG_CHECK_FINITE = 2,   /* scan x for NaN/Inf first and fail with TT_ERR_NONFINITE */
  TT_FLAG_NO_FOLD = 4,        /* materialise full-rank steps instead of folding their rotation */
  TT_FLAG_IDENTITY_GAUGE = 8, /* full-rank steps keep the identity basis (no Gram pass) */
  TT_FLAG_KEEP_SIGMA = 16,    /* fill tt_stats.sigma */
  TT_FLAG_PROFILE = 32,       /* time the bulk passes over the largest unfolding (tt_stats.top_*) */
  /* eps > 0 only.  Plain adaptive EDrSVD: the sketch width of a randomized step starts at
   * 16 + s and doubles (up to r + s, r the caller's rank bound) until the a-posteriori error
   * estimate ||A||^2 - ||Q^T A||^2 meets the step tolerance. */
  TT_FLAG_ADAPTIVE_KS = 64,
  /* eps > 0 only.  Learned EDrSVD: the context's predictor (tt_ctx_set_predictor) chooses
   * rank, oversampling and power iterations of each randomized step from Gaussian-probe
   * features (tt_probe_features); when the a-posteriori estimate of that attempt exceeds the
   * step tolerance the plain adaptive EDrSVD takes over from twice its sketch width (at least
 * the plain method's first width). */
  TT_FLAG_LEARNED = 128,
  /* x is a host pointer (pinned memory recommended) that is never copied whole to the device:
   * the passes over the first unfolding (its Gram and its projection) stream it in column
   * chunks (tt_ctx_set_stream_chunk) through two device buffers, the copy of chunk c + 1
   * overlapping the kernels of chunk c; the rest of the chain runs on the projected data.  For
   * tensors larger than device memory whose first unfolding has at most TT_MAX_SMALL rows and
   * whose projected data (r1 x n2...nd) fits.  TT-SVD with fixed ranks; cores are device
   * pointers unless TT_FLAG_HOST_IO is also set.  Replaces ttdec_half_lu_host_6
   * (ttdecomposition/high_order_GPUs/ttdec6_singleGPU.cu:656-796; its per-slice Gram at :567
   * restarts the accumulation with beta = 0 on every slice, here the slices are summed). */
  TT_FLAG_HOST_STREAM = 256,
  /* eps > 0: fail with TT_ERR_RANK when a rank bound keeps the error above eps
   * (tt_stats.eps_unmet > 0) instead of returning TT_OK with est_rel_err > eps. */
  TT_FLAG_STRICT_EPS = 512
};

typedef struct tt_opts {
  int method;            /* TT_METHOD_* */
  int gemm;              /* TT_GEMM_* */
  int oversample;        /* s: sketch width is r + s (reference: s = 8, ablation edrsvd_GPU:347) */
  int power_iters;       /* p (reference: p = 1) */
  unsigned long long seed;
  double eps;            /* relative tolerance; 0 = fixed ranks (the reference accepts eps but ignores it) */
  int flags;             /* TT_FLAG_* */
  int max_sweeps;        /* Jacobi sweep limit (0 = default 40) */
} tt_opts;

#define TT_STATS_MAX_SIGMA 64
typedef struct tt_stats {
  double ms;                                   /* device time of the call (CUDA events) */
  int nsteps;                                  /* unfoldings factorised */
  int ranks[TT_MAX_ORDER + 1];                 /* ranks used (after clamping / adaptation) */
  int nsigma[TT_MAX_ORDER];                    /* singular values stored per unfolding */
  float sigma[TT_MAX_ORDER][TT_STATS_MAX_SIGMA];
  int jacobi_sweeps;                           /* largest sweep count of any eigen-solve */
  int kernels;                                 /* kernels launched by the call */
  double est_rel_err;                          /* eps > 0: sqrt(discarded energy / ||X||^2) */
  double flops;                                /* algorithmic FLOPs of the bulk GEMM passes executed */
  double bytes;                                /* algorithmic HBM bytes of those passes (operands once) */
  /* TT_FLAG_PROFILE: per pass kind (TT_PASS_*), summed device time (CUDA events on the
   * context stream around each launch), algorithmic bytes moved and launch count. */
  double pass_ms[4];
  double pass_bytes[4];
  int pass_launches[4];
  /* TT_FLAG_PROFILE: the single longest bulk pass of the call (kind, unfolding index,
   * device time, algorithmic bytes). */
  int top_kind;
  int top_step;
  double top_ms;
  double top_bytes;
  int passes;                      /* bulk passes over unfoldings (Gram, sketch, projection, probe) */
  int fallbacks;                   /* TT_FLAG_LEARNED: steps the plain adaptive EDrSVD took over */
  int step_ks[TT_MAX_ORDER];       /* sketch width finally used per unfolding (0: exact step) */
  int step_power[TT_MAX_ORDER];    /* power iterations finally used per unfolding */
  int step_attempts[TT_MAX_ORDER]; /* EDrSVD attempts per unfolding */
  /* eps > 0: unfoldings whose rank bound (the caller's rank, or the sketch-width limit
   * TT_MAX_SMALL of a randomized step) stopped the truncation with more than the step's
   * budget delta^2 = eps^2 ||X||^2 / (d - 1) discarded.  Nonzero means est_rel_err > eps: the
   * tolerance was not met (the call still returns TT_OK with the best decomposition within
   * the bounds; TT_FLAG_STRICT_EPS turns this into TT_ERR_RANK). */
  int eps_unmet;
} tt_stats;

/* Bulk pass kinds reported in tt_stats.pass_*. */
enum { TT_PASS_GRAM = 0, TT_PASS_SKETCH = 1, TT_PASS_PROJECT = 2, TT_PASS_OTHER = 3 };

typedef struct tt_ctx tt_ctx;

/* Context: one device, one stream, a growing device workspace.  Not thread-safe per
 * context; use one context per host thread.  Replaces the per-call cublasCreate /
 * cusolverDnCreate of the reference (ttdec6_singleGPU.cu:808-815). */
int tt_ctx_create(tt_ctx** out, int device, void* stream);
int tt_ctx_destroy(tt_ctx* ctx);
int tt_ctx_set_stream(tt_ctx* ctx, void* stream);
int tt_ctx_reserve(tt_ctx* ctx, size_t bytes);
/* Fault injection and limits (no counterpart in the reference, which asserts on every CUDA
 * status).  tt_ctx_set_alloc_limit: workspace growth above `bytes` fails with TT_ERR_NOMEM as
 * if cudaMalloc had failed (0 removes the limit).  tt_ctx_set_wait_limit: wall-clock limit of
 * every pipeline wait of the TMA kernels on the context's device (ns; 0 = the default 2 s); a
 * wait that runs out ends its kernel with TT_ERR_TIMEOUT after the CTA has drained its own
 * copies (the drain always gets 2 s).  tt_k_wait_selftest: a kernel waiting on a barrier that
 * nothing completes, under the same limit; returns TT_ERR_TIMEOUT. */
int tt_ctx_set_alloc_limit(tt_ctx* ctx, size_t bytes);
int tt_ctx_set_wait_limit(tt_ctx* ctx, unsigned long long ns);
int tt_k_wait_selftest(tt_ctx* ctx);

/* Bytes of one host-streaming chunk (TT_FLAG_HOST_STREAM; default 256 MiB, minimum one column). */
int tt_ctx_set_stream_chunk(tt_ctx* ctx, size_t bytes);
const char* tt_last_error(void);
void tt_default_opts(tt_opts* o);
int tt_abi_version(void);

/* Order-d TT-SVD with fixed ranks r[0..d] (r[0] = r[d] = 1).  cores[k] receives the
 * column-major (r[k], n[k], r[k+1]) core.  Ranks larger than an unfolding can carry are
 * zero-padded.  Replaces ttdec_half_lu_device_6 (ttdecomposition/high_order_GPUs/
 * ttdec6_singleGPU.cu:799) and the order-3 ttdec_gpu_float (ttdecomposition/
 * third_order_GPUs/opt/ttdec_gpu_float_rsvd_lu_half.cu:778), which discard their cores. */
int tt_svd(tt_ctx* ctx, const float* x, int d, const int* n, const int* r, const tt_opts* opts,
           float* const* cores, tt_stats* stats);

/* Order-d TR-SVD with bond ranks r[0..d], r[0] = r[d].  Step 1 factorises unfolding 1 at
 * rank r0*r1 (zero-padded beyond n1) and permutes (r0, r1, N) -> (r1, N, r0).  cores[k]
 * receives the column-major (r[k], n[k], r[k+1]) ring core.  Replaces the TR
 * ttdec_half_lu_device_6 (trdecomposition/high_order_GPUs/trdec6_singleGPU.cu:827) and
 * trdec_gpu_float (trdecomposition/third_order_GPU/opt_GPU/trdec_gpu_float_rsvd_lu_half.cu:734). */
int tr_svd(tt_ctx* ctx, const float* x, int d, const int* n, const int* r, const tt_opts* opts,
           float* const* cores, tt_stats* stats);

/* Relative reconstruction error ||X - TT(cores)||_F / ||X||_F computed on the device with
 * FP64 accumulation; ring = 1 for TR cores.  Replaces calMSE / norm2HH
 * (ttdecomposition/high_order_GPUs/ttdec6_singleGPU.cu:122-182), a serial host loop that
 * also overwrote the input. */
int tt_rel_error(tt_ctx* ctx, const float* x, int d, const int* n, const int* r, int ring,
                 const float* const* cores, double* rel_err);

/* ---- building blocks (device pointers, stream-ordered on the context's stream) ---- */

/* Gaussian N(0,1) column-major (rows x cols, leading dim ld) matrix from Philox4x32-10.
 * Replaces curandGenerateNormal (ttdec_gpu_float_rsvd_lu_half.cu:585-587). */
int tt_k_gaussian(tt_ctx* ctx, float* out, long long rows, int cols, long long ld,
                  unsigned long long seed, unsigned stream_id);

/* Rows [row0, row0 + nrows) of the Gaussian matrix tt_k_gaussian makes with total_rows rows
 * (same seed / stream): the Omega block of one rank's columns in a column-sharded EDrSVD.
 * No counterpart in the reference (single GPU per unfolding). */
int tt_k_gaussian_rows(tt_ctx* ctx, float* out, long long row0, long long nrows, long long total_rows, int cols,
                       long long ld, unsigned long long seed, unsigned stream_id);

/* Sketch Y = A * W: A (m x n, lda = m), W (n x N, ldw), Y (m x N, FP64, ldy = m).
 * Replaces GemmEx Y = A*Omega / Y = A*Q (ttdec_gpu_float_rsvd_lu_half.cu:601-619,657-675). */
int tt_k_sketch(tt_ctx* ctx, const float* a, long long m, long long n, const float* w, int N,
                long long ldw, double* y, int gemm);

/* Projection out = A^T * Q: A (m x n, lda = m), Q (m x N, ldq), out row-major n x N with
 * row stride ldo (i.e. the column-major N x n matrix Q^T A).  Replaces GemmEx B = Q^T A
 * and Z = A^T Q (ttdec_gpu_float_rsvd_lu_half.cu:631-649,690-708; ttdec6_singleGPU.cu:424-488). */
int tt_k_project(tt_ctx* ctx, const float* a, long long m, long long n, const float* q, int N,
                 long long ldq, float* out, long long ldo, int gemm);

/* Gram of the rows W = A * A^T (m x m, FP64), A (m x n, lda = m), m <= TT_MAX_SMALL.
 * gemm = TT_GEMM_TC uses tcgen05 TF32 tiles (operands rounded to nearest by the TMA unit,
 * FP32 accumulation, FP64 across blocks); TT_GEMM_FP32 the FP32 FMA kernel.  With
 * TT_GEMM_AUTO or TT_GEMM_FP32, m <= 32 (m % 4 == 0) takes the exact CUDA-core kernel (FP32
 * products, FP64 sums), the one every decomposition uses for such unfoldings.
 * Replaces largeMatrixSelfMulti_once_device (ttdec6_singleGPU.cu:388-401). */
int tt_k_gram_rows(tt_ctx* ctx, const float* a, long long m, long long n, double* w, int gemm);

/* Gram of a tall matrix W = Z^T Z (N x N, FP64): Z is n x N with element (j, c) at
 * z[j*rs + c*cs] (column-major: rs = 1, cs = ld; row-major: rs = ld, cs = 1). */
int tt_k_gram_tall(tt_ctx* ctx, const float* z, long long n, int N, long long rs, long long cs,
                   double* w);

/* CholeskyQR2 in place on a tall FP32 matrix Y (n x N, column-major, ld): Y <- Q, R (N x N,
 * FP64, upper) optional.  Columns that are numerically dependent are zeroed.  Replaces
 * basicQR = geqrf + orgqr (ttdec_gpu_float_rsvd_lu_half.cu:85-159). */
int tt_k_cholqr2(tt_ctx* ctx, float* y, long long n, int N, long long ld, double* r);

/* Symmetric eigen-decomposition of W (N x N, FP64, column-major) by parallel cyclic
 * Jacobi in shared memory; eigenvalues descending, eigenvectors as columns.  Replaces
 * cusolverDnSsyevd + matrixInvertColumn (ttdec6_singleGPU.cu:274-290,334-385). */
int tt_k_syev(tt_ctx* ctx, const double* w, int N, double* evals, double* evecs, int* sweeps);


/* Allocation-free sketch Y = A * W (same operands and result as tt_k_sketch), for callers
 * that cannot call cudaMalloc: a process whose device memory belongs to another allocator or
 * a pre-reserved arena, or a latency-critical loop that must not let cudaMalloc synchronise
 * the device.  No context is needed; the call allocates nothing.  The kernel's split-K
 * scratch is one static device array of 2^21 doubles (16 MiB, held by every GPU that loads
 * the library until exit); m * N above 2^21 - 32 is rejected with TT_ERR_SHAPE.  All calls
 * share that array: calls that overlap on the GPU race and must be serialised.  The first
 * call on a device looks up the array's address (with that device current) and should come
 * before any stream capture.  Runs on `stream` (NULL = legacy default stream), which must
 * belong to the current device (TT_ERR_ARG otherwise), and returns after the result is
 * complete.  gemm outside TT_GEMM_AUTO..TT_GEMM_FP32 is rejected with TT_ERR_ARG.  This entry point has no counterpart in the reference. */
int tt_k_sketch_noalloc(const float* a, long long m, long long n, const float* w, int N,
                        long long ldw, double* y, int gemm, void* stream);

/* Batched TT-SVD of many small tensors in one persistent launch (one CTA per tensor at a
 * time, a work counter spreads the tensors over the SMs).  `n` holds count x d mode sizes,
 * `x` the packed column-major tensors at element offsets `x_off`; all host arrays except x and
 * cores (device).  eps > 0: delta-truncation per tensor as in tt_svd (ranks capped by rmax);
 * eps = 0: ranks min(rmax, unfolding size).  rmax <= 32; unfoldings whose small side exceeds
 * 32 are sketched (EDrSVD with `oversample`, Philox `seed`) and may have at most 512 rows.
 * Cores of tensor t are written compactly from element core_off[t] (core k after core k-1,
 * each column-major (r_k, n_k, r_{k+1})); tt_batch_core_capacity gives the room one tensor
 * needs.  ranks receives count x (d + 1) ranks, err_est (optional) the per-tensor error bound
 * sqrt(discarded energy / ||X||^2).  No counterpart in the reference (one tensor per call). */
int tt_svd_batched(tt_ctx* ctx, int count, int d, const int* n, const float* x, const long long* x_off,
                   double eps, int rmax, int oversample, unsigned long long seed, float* cores,
                   const long long* core_off, int* ranks, double* err_est);
long long tt_batch_core_capacity(int d, const int* n, int rmax);

/* Batch plans: the same decomposition as tt_svd_batched for a batch that is run repeatedly.
 * tt_batch_plan_create validates the shapes once and keeps the shape table, a largest-first
 * work order and the kernel scratch on the device (own allocation and stream; inputs are
 * ordered after the context stream's prior work).  tt_batch_plan_tune times every variant
 * (sketch chunk width 16 / 32 / 64 x natural or largest-first work order; `reps` launches
 * each, ms_out receives the 6 averages or may be NULL) on the caller's batch and keeps the
 * fastest; otherwise chunk 32, largest-first.  tt_batch_plan_run replays the launch sequence
 * (status and work-counter reset, the persistent kernel, read-back of ranks / error estimates)
 * as one CUDA graph, captured on the first run and again when x, cores or the variant change;
 * ranks and err_est as in tt_svd_batched (host arrays, may be NULL). */
typedef struct tt_batch_plan tt_batch_plan;
int tt_batch_plan_create(tt_ctx* ctx, int count, int d, const int* n, const long long* x_off, double eps, int rmax,
                         int oversample, unsigned long long seed, const long long* core_off, tt_batch_plan** plan);
int tt_batch_plan_tune(tt_batch_plan* plan, const float* x, float* cores, int reps, float* ms_out);
int tt_batch_plan_variant(const tt_batch_plan* plan, int* chunk, int* largest_first);
int tt_batch_plan_run(tt_batch_plan* plan, const float* x, float* cores, int* ranks, double* err_est);
int tt_batch_plan_destroy(tt_batch_plan* plan);

/* Learned EDrSVD parameters.  A 8 -> 64 -> 64 -> 3 ReLU network maps the probe features of
 * an unfolding to (log2 rank / 10, log2 oversampling / 5, power iterations / 2); it is trained
 * by the library's own kernels (tt_mlp_train) on labels of the plain method.  All pointers
 * are device pointers unless stated.  No counterpart in the reference, whose EDrSVD takes
 * fixed s and p (ttdecomposition/third_order_GPUs/opt/ttdec_gpu_float_rsvd_lu_half.cu:797-798). */
/* Install (host params, TT_MLP_PARAMS floats) or clear (NULL) the predictor of TT_FLAG_LEARNED. */
int tt_ctx_set_predictor(tt_ctx* ctx, const float* params);
/* Features of the (m x n) unfolding a: a Gaussian probe Y = A Omega with TT_PROBE_COLS columns
 * (Philox `seed`, stream `stream_id`), the eigenvalues mu of Y^T Y, and
 * [log2(min(m,n))/10, log10(mu_j/mu_1)/4 for j = 2,4,8,12,16, log10(16 E/mu_1)/4, log10(tol)/4]
 * with E = ||A||_F^2 (`energy`; computed when < 0) and `tol` the step's relative tolerance. */
int tt_probe_features(tt_ctx* ctx, const float* a, long long m, long long n, double energy, double tol,
                      unsigned long long seed, unsigned stream_id, float* features);
/* y (n x 3, row-major) = network(x (n x 8, row-major)). */
int tt_mlp_forward(tt_ctx* ctx, const float* params, const float* x, int n, float* y);
/* Gradient (TT_MLP_PARAMS floats) and value (1 float, may be NULL) of the mean over the n
 * samples of the summed squared output error against t (n x 3). */
int tt_mlp_grad(tt_ctx* ctx, const float* params, const float* x, const float* t, int n, float* grad, float* loss);
/* `steps` Adam steps (lr, beta 0.9 / 0.999, bias-corrected from step step0 + 1) on minibatches
 * of `batch` samples drawn with replacement from the n samples (Philox `seed`); params,
 * adam_m and adam_v are updated in place; loss_trace (steps floats, may be NULL) receives
 * each minibatch's loss before its update.  One persistent single-CTA launch. */
int tt_mlp_train(tt_ctx* ctx, float* params, float* adam_m, float* adam_v, const float* x, const float* t, int n,
                 int steps, int batch, float lr, int step0, unsigned long long seed, float* loss_trace);

/* Core files.  The reference frees its cores before returning (ttdec6_singleGPU.cu:947-952)
 * and has no file format; this one stores a decomposition for later use.  Layout
 * (little-endian): 8-byte magic "TTRCORE1", int32 kind (0 = TT, 1 = TR), int32 d,
 * int32 dtype (0 = FP32), int32 reserved (0), int64 n[d], int64 r[d+1], then core k as
 * r[k] * n[k] * r[k+1] FP32 values, column-major (r[k], n[k], r[k+1]).  `device` = 1 when
 * the core pointers are device memory (copied through the host). */
int tt_cores_save(const char* path, int d, const int* n, const int* r, int ring,
                  const float* const* cores, int device);
/* Reads the header: d, n[0..d-1], r[0..d] (arrays of TT_MAX_ORDER and TT_MAX_ORDER + 1 ints)
 * and ring (0/1). */
int tt_cores_header(const char* path, int* d, int* n, int* r, int* ring);
/* Reads the cores into caller buffers sized from tt_cores_header. */
int tt_cores_load(const char* path, float* const* cores, int device);

/* TR bond permute (r0, r1, N) -> (r1, N, r0), column-major.  Replaces tensorToMode231
 * (trdecomposition/high_order_GPUs/trdec6_singleGPU.cu:49-58). */
int tt_k_permute231(tt_ctx* ctx, const float* in, float* out, int r0, int r1, long long n);

/* Reference-compatible entry points with pointer arguments (the C++ overloads with the
 * reference's exact signatures are declared in ttrsvd_ref.h).  Return elapsed seconds
 * (negative on failure), like the reference. */
float tt_ref_ttdec_gpu_float(float* h_tensor, int* h_n_array, int* h_r_array, double* eps,
                             float* single_error, float* single_com_ratio);
float tt_ref_trdec_gpu_float(float* h_tensor, int* h_n_array, int* h_r_array, double* eps,
                             float* single_error, float* single_com_ratio);
float tt_ref_ttdec_half_lu_device_6(float* h_a, const int* tt_ranks, const int* tt_demns,
                                    int calculate_times, int p, int cal_error);
float tt_ref_trdec_half_lu_device_6(float* h_a, const int* tt_ranks, const int* tt_demns,
                                    int calculate_times, int p, int cal_error);
/* ttdec_half_lu_host_6 (ttdec6_singleGPU.cu:656): host-streamed first unfolding in p slices. */
float tt_ref_ttdec_half_lu_host_6(float* h_a, const int* tt_ranks, const int* tt_demns,
                                  int calculate_times, int p, int cal_error);

#ifdef __cplusplus
}
#endif
#endif /* TTRSVD_H */
