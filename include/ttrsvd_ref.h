/*
 * ttrsvd_ref.h - C++ entry points with the reference programs' exact host signatures.
 *
 * A reference benchmark main (e.g. ttdecomposition/third_order_GPUs/opt/main.cpp) links
 * against libttrsvd.so instead of its own .cu file and calls the same function.  Each
 * returns the elapsed seconds of one decomposition (mean over calculateTimes for order 6);
 * the input tensor is a caller-owned column-major host buffer and is never modified.
 */
#ifndef TTRSVD_REF_H
#define TTRSVD_REF_H

#include "ttrsvd.h"

#ifdef __cplusplus
/* ttdecomposition/third_order_GPUs/opt/func.h:16 (definition ttdec_gpu_float_rsvd_lu_half.cu:778).
 * eps is accepted and ignored, as in the reference.  singleError, when non-null, receives
 * ||X - X^||/||X||; singleComRatio receives the core-to-tensor size ratio. */
float ttdec_gpu_float(float* h_tensor, int* h_n_array, int* h_r_array, double* eps,
                      float* singleError, float* singleComRatio);

/* trdecomposition/third_order_GPU/opt_GPU/func.h:15 (definition trdec_gpu_float_rsvd_lu_half.cu:734);
 * h_r_array = {r0, r1, r2, r0}. */
float trdec_gpu_float(float* h_tensor, int* h_n_array, int* h_r_array, double* eps,
                      float* singleError, float* singleComRatio);

/* ttdecomposition/high_order_GPUs/ttdec6_singleGPU.cu:799.  p (projection slices) is accepted
 * and ignored.  With calError the reference's "MSE:" line is printed. */
float ttdec_half_lu_device_6(float* h_A, const int* ttRanks, const int* ttDemns,
                             const int& calculateTimes, const int& p, bool calError);

/* ttdecomposition/high_order_GPUs/ttdec6_singleGPU.cu:656: the tensor stays in (ideally pinned)
 * host memory and its first unfolding is streamed in p column slices, copies overlapped with
 * the kernels (TT_FLAG_HOST_STREAM; first unfolding of at most TT_MAX_SMALL rows).  The
 * reference restarts its Gram accumulation on every slice (beta = 0, ttdec6_singleGPU.cu:567);
 * here the slices are summed.  calError prints the "MSE:" line. */
float ttdec_half_lu_host_6(float* h_A, int* ttRanks, const int* ttDemns, const int& calculateTimes, const int& p,
                           const bool calError);

/* trdecomposition/high_order_GPUs/trdec6_singleGPU.cu:827, where the TR program reuses the
 * name ttdec_half_lu_device_6; exported here as trdec_half_lu_device_6 so both can share one
 * library.  ttRanks = {r0, r1, ..., r5, r0}. */
float trdec_half_lu_device_6(float* h_A, const int* ttRanks, const int* ttDemns,
                             const int& calculateTimes, const int& p, bool calError);
#endif

#endif /* TTRSVD_REF_H */
