"""ctypes binding of libttrsvd.so (declarations mirror include/ttrsvd.h)."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libttrsvd.so")

TT_OK = 0
STATUS_NAMES = {
    0: "TT_OK", 1: "TT_ERR_ARG", 2: "TT_ERR_SHAPE", 3: "TT_ERR_RANK", 4: "TT_ERR_NONFINITE",
    5: "TT_ERR_NOMEM", 6: "TT_ERR_NOCONV", 7: "TT_ERR_TIMEOUT", 8: "TT_ERR_CUDA",
    9: "TT_ERR_UNSUPPORTED", 10: "TT_ERR_IO",
}
TT_GEMM_AUTO, TT_GEMM_TC, TT_GEMM_FP32 = 0, 1, 2
TT_METHOD_EDRSVD, TT_METHOD_EXACT = 0, 1
TT_FLAG_HOST_IO, TT_FLAG_CHECK_FINITE, TT_FLAG_NO_FOLD, TT_FLAG_IDENTITY_GAUGE, TT_FLAG_KEEP_SIGMA = 1, 2, 4, 8, 16
TT_FLAG_PROFILE = 32
TT_FLAG_ADAPTIVE_KS, TT_FLAG_LEARNED, TT_FLAG_HOST_STREAM, TT_FLAG_STRICT_EPS = 64, 128, 256, 512
TT_MLP_INPUTS, TT_MLP_OUTPUTS, TT_MLP_PARAMS, TT_PROBE_COLS = 8, 3, 4931, 16
TT_PASS_GRAM, TT_PASS_SKETCH, TT_PASS_PROJECT, TT_PASS_OTHER = 0, 1, 2, 3
PASS_NAMES = ["gram", "sketch", "project", "other"]
TT_MAX_ORDER = 16
TT_MAX_SMALL = 128
TT_STATS_MAX_SIGMA = 64

# Every extern "C" symbol declared in include/ttrsvd.h.
EXPORTED = [
    "tt_ctx_create", "tt_ctx_destroy", "tt_ctx_set_stream", "tt_ctx_reserve", "tt_ctx_set_stream_chunk", "tt_ctx_set_alloc_limit", "tt_ctx_set_wait_limit", "tt_k_wait_selftest",
    "tt_last_error",
    "tt_default_opts", "tt_abi_version", "tt_svd", "tr_svd", "tt_rel_error", "tt_k_gaussian", "tt_k_gaussian_rows",
    "tt_k_sketch", "tt_k_project", "tt_k_gram_rows", "tt_k_gram_tall", "tt_k_cholqr2",
    "tt_k_syev", "tt_k_sketch_noalloc", "tt_svd_batched", "tt_batch_core_capacity",
    "tt_batch_plan_create", "tt_batch_plan_tune", "tt_batch_plan_variant", "tt_batch_plan_run",
    "tt_batch_plan_destroy",
    "tt_cores_save", "tt_cores_header", "tt_cores_load",
    "tt_ctx_set_predictor", "tt_probe_features", "tt_mlp_forward", "tt_mlp_grad", "tt_mlp_train",
    "tt_k_permute231", "tt_ref_ttdec_gpu_float", "tt_ref_trdec_gpu_float",
    "tt_ref_ttdec_half_lu_device_6", "tt_ref_trdec_half_lu_device_6", "tt_ref_ttdec_half_lu_host_6",
]


class TTOpts(C.Structure):
    _fields_ = [
        ("method", C.c_int), ("gemm", C.c_int), ("oversample", C.c_int), ("power_iters", C.c_int),
        ("seed", C.c_ulonglong), ("eps", C.c_double), ("flags", C.c_int), ("max_sweeps", C.c_int),
    ]


class TTStats(C.Structure):
    _fields_ = [
        ("ms", C.c_double), ("nsteps", C.c_int), ("ranks", C.c_int * (TT_MAX_ORDER + 1)),
        ("nsigma", C.c_int * TT_MAX_ORDER),
        ("sigma", (C.c_float * TT_STATS_MAX_SIGMA) * TT_MAX_ORDER),
        ("jacobi_sweeps", C.c_int), ("kernels", C.c_int), ("est_rel_err", C.c_double),
        ("flops", C.c_double), ("bytes", C.c_double), ("pass_ms", C.c_double * 4),
        ("pass_bytes", C.c_double * 4), ("pass_launches", C.c_int * 4),
        ("top_kind", C.c_int), ("top_step", C.c_int), ("top_ms", C.c_double), ("top_bytes", C.c_double),
        ("passes", C.c_int), ("fallbacks", C.c_int), ("step_ks", C.c_int * TT_MAX_ORDER),
        ("step_power", C.c_int * TT_MAX_ORDER), ("step_attempts", C.c_int * TT_MAX_ORDER),
        ("eps_unmet", C.c_int),
    ]


class TTError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libttrsvd.so; raise if it was not built (there is no fallback implementation)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m tensor_train_ring_decompositions_hpc_gpu_b200.build`")
    lib = C.CDLL(LIB_PATH)
    vp, i, ll, ull, d = C.c_void_p, C.c_int, C.c_longlong, C.c_ulonglong, C.c_double
    P = C.POINTER
    sig = {
        "tt_ctx_create": (i, [P(vp), i, vp]),
        "tt_ctx_destroy": (i, [vp]),
        "tt_ctx_set_stream": (i, [vp, vp]),
        "tt_ctx_reserve": (i, [vp, C.c_size_t]),
        "tt_ctx_set_stream_chunk": (i, [vp, C.c_size_t]),
        "tt_ctx_set_alloc_limit": (i, [vp, C.c_size_t]),
        "tt_ctx_set_wait_limit": (i, [vp, C.c_ulonglong]),
        "tt_k_wait_selftest": (i, [vp]),
        "tt_last_error": (C.c_char_p, []),
        "tt_default_opts": (None, [P(TTOpts)]),
        "tt_abi_version": (i, []),
        "tt_svd": (i, [vp, vp, i, P(i), P(i), P(TTOpts), P(vp), P(TTStats)]),
        "tr_svd": (i, [vp, vp, i, P(i), P(i), P(TTOpts), P(vp), P(TTStats)]),
        "tt_rel_error": (i, [vp, vp, i, P(i), P(i), i, P(vp), P(d)]),
        "tt_k_gaussian": (i, [vp, vp, ll, i, ll, ull, C.c_uint]),
        "tt_k_sketch": (i, [vp, vp, ll, ll, vp, i, ll, vp, i]),
        "tt_k_project": (i, [vp, vp, ll, ll, vp, i, ll, vp, ll, i]),
        "tt_k_gram_rows": (i, [vp, vp, ll, ll, vp, i]),
        "tt_k_gram_tall": (i, [vp, vp, ll, i, ll, ll, vp]),
        "tt_k_cholqr2": (i, [vp, vp, ll, i, ll, vp]),
        "tt_k_syev": (i, [vp, vp, i, vp, vp, P(i)]),
        "tt_k_permute231": (i, [vp, vp, vp, i, i, ll]),
        "tt_k_sketch_noalloc": (i, [vp, ll, ll, vp, i, ll, vp, i, vp]),
        "tt_k_gaussian_rows": (i, [vp, vp, ll, ll, ll, i, ll, ull, C.c_uint]),
        "tt_svd_batched": (i, [vp, i, i, P(i), vp, P(ll), d, i, i, C.c_ulonglong, vp, P(ll), P(i), P(d)]),
        "tt_batch_core_capacity": (ll, [i, P(i), i]),
        "tt_batch_plan_create": (i, [vp, i, i, P(i), P(ll), d, i, i, ull, P(ll), P(vp)]),
        "tt_batch_plan_tune": (i, [vp, vp, vp, i, P(C.c_float)]),
        "tt_batch_plan_variant": (i, [vp, P(i), P(i)]),
        "tt_batch_plan_run": (i, [vp, vp, vp, P(i), P(d)]),
        "tt_batch_plan_destroy": (i, [vp]),
        "tt_ctx_set_predictor": (i, [vp, vp]),
        "tt_probe_features": (i, [vp, vp, ll, ll, d, d, ull, C.c_uint, vp]),
        "tt_mlp_forward": (i, [vp, vp, vp, i, vp]),
        "tt_mlp_grad": (i, [vp, vp, vp, vp, i, vp, vp]),
        "tt_mlp_train": (i, [vp, vp, vp, vp, vp, vp, i, i, i, C.c_float, i, ull, vp]),
        "tt_cores_save": (i, [C.c_char_p, i, P(i), P(i), i, P(vp), i]),
        "tt_cores_header": (i, [C.c_char_p, P(i), P(i), P(i), P(i)]),
        "tt_cores_load": (i, [C.c_char_p, P(vp), i]),
        "tt_ref_ttdec_gpu_float": (C.c_float, [vp, P(i), P(i), P(d), P(C.c_float), P(C.c_float)]),
        "tt_ref_trdec_gpu_float": (C.c_float, [vp, P(i), P(i), P(d), P(C.c_float), P(C.c_float)]),
        "tt_ref_ttdec_half_lu_device_6": (C.c_float, [vp, P(i), P(i), i, i, i]),
        "tt_ref_trdec_half_lu_device_6": (C.c_float, [vp, P(i), P(i), i, i, i]),
        "tt_ref_ttdec_half_lu_host_6": (C.c_float, [vp, P(i), P(i), i, i, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int):
    if code != TT_OK:
        msg = load().tt_last_error()
        raise TTError(code, msg.decode() if msg else "")
    return code


def int_array(vals):
    arr = (C.c_int * len(vals))(*[int(v) for v in vals])
    return arr
