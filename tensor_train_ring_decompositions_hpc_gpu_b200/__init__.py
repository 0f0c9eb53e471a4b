"""B200-native TT-SVD / TR-SVD (EDrSVD per unfolding) over the C ABI of libttrsvd.so.

Tensors follow the reference's storage convention: column-major, mode 1 fastest.  Device
tensors are torch CUDA tensors (torch supplies device memory and the current stream);
host tensors are NumPy arrays.  Every decomposition runs in the hand-written sm_100a
kernels of libttrsvd.so; when the library is missing, importing the compute functions
raises instead of falling back to anything else.

Reference-compatible entry points (same names, argument meaning and return value):
``ttdec_gpu_float``, ``trdec_gpu_float`` (order 3) and ``ttdec_half_lu_device_6``,
``trdec_half_lu_device_6`` (order 6).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (TT_FLAG_ADAPTIVE_KS, TT_FLAG_CHECK_FINITE, TT_FLAG_HOST_IO, TT_FLAG_HOST_STREAM,
                   TT_FLAG_IDENTITY_GAUGE,
                   TT_FLAG_KEEP_SIGMA, TT_FLAG_LEARNED, TT_FLAG_NO_FOLD, TT_FLAG_STRICT_EPS, TT_GEMM_AUTO, TT_GEMM_FP32, TT_GEMM_TC,
                   TT_METHOD_EDRSVD, TT_METHOD_EXACT, TTError, check)

__all__ = [
    "tt_svd", "tr_svd", "rel_error", "Result", "gaussian", "sketch", "project", "gram_rows",
    "gram_tall", "cholqr2", "syev", "permute231", "ttdec_gpu_float", "trdec_gpu_float",
    "ttdec_half_lu_device_6", "trdec_half_lu_device_6", "TTError", "lib", "GEMM", "METHOD",
    "set_predictor", "probe_features", "mlp_forward", "mlp_grad", "mlp_train", "set_stream_chunk",
]

GEMM = {"auto": TT_GEMM_AUTO, "tc": TT_GEMM_TC, "fp32": TT_GEMM_FP32}
METHOD = {"edrsvd": TT_METHOD_EDRSVD, "exact": TT_METHOD_EXACT}


def lib():
    return _lib.load()


def _torch():
    import torch
    return torch


class _Ctx:
    def __init__(self, device: int):
        self.device = device
        self.ptr = C.c_void_p()
        check(lib().tt_ctx_create(C.byref(self.ptr), device, None))

    def bind(self, stream_handle):
        check(lib().tt_ctx_set_stream(self.ptr, C.c_void_p(stream_handle)))
        return self.ptr

    def __del__(self):
        try:
            if self.ptr:
                lib().tt_ctx_destroy(self.ptr)
        except Exception:
            pass


_CTX: dict = {}


def _ctx_for(device: int | None = None, stream=None):
    torch = _torch()
    if device is None:
        device = torch.cuda.current_device()
    if device not in _CTX:
        _CTX[device] = _Ctx(device)
    ctx = _CTX[device]
    if stream is None:
        stream = torch.cuda.current_stream(device)
    return ctx.bind(stream.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _fortran_buffer(x):
    """Column-major flat device buffer of a torch tensor given in logical index order."""
    torch = _torch()
    d = x.dim()
    buf = x.permute(*reversed(range(d))).contiguous() if d > 1 else x.contiguous()
    if buf.dtype != torch.float32:
        buf = buf.float()
    return buf


def _core_view(flat, r0, n, r1):
    """Logical (r0, n, r1) view of a column-major core buffer."""
    return flat.view(r1, n, r0).permute(2, 1, 0)


@dataclass
class Result:
    cores: list
    ms: float = 0.0
    sigmas: list = field(default_factory=list)
    ranks: list = field(default_factory=list)
    kernels: int = 0
    jacobi_sweeps: int = 0
    est_rel_err: float = 0.0
    passes: int = 0
    fallbacks: int = 0
    step_ks: list = field(default_factory=list)
    step_power: list = field(default_factory=list)
    step_attempts: list = field(default_factory=list)
    eps_unmet: int = 0  # eps > 0: unfoldings whose rank bound kept the discarded energy above budget
    flops: float = 0.0  # arithmetic of the passes the library ran (its own pass accounting)


def _opts(gemm, method, oversample, power_iters, seed, flags, max_sweeps):
    o = _lib.TTOpts()
    lib().tt_default_opts(C.byref(o))
    o.gemm = GEMM[gemm] if isinstance(gemm, str) else int(gemm)
    o.method = METHOD[method] if isinstance(method, str) else int(method)
    o.oversample = int(oversample)
    o.power_iters = int(power_iters)
    o.seed = int(seed)
    o.flags = int(flags) | TT_FLAG_KEEP_SIGMA
    o.max_sweeps = int(max_sweeps)
    return o


def set_stream_chunk(nbytes, device=None):
    """Chunk size (bytes) of the host-streamed first unfolding (tt_svd(..., stream=True))."""
    check(lib().tt_ctx_set_stream_chunk(_ctx_for(device), int(nbytes)))


def _run(ring: bool, x, ranks, gemm="auto", method="edrsvd", oversample=8, power_iters=0,
         seed=1234, flags=0, max_sweeps=40, shape=None, eps=0.0, stream=False):
    ranks = [int(r) for r in ranks]
    host = isinstance(x, np.ndarray)
    if stream:
        if not host:
            raise ValueError("stream=True takes a host (NumPy) tensor, ideally backed by pinned memory")
        flags |= TT_FLAG_HOST_STREAM
    if host:
        xa = x if (x.dtype == np.float32 and x.flags.f_contiguous) else np.asfortranarray(x, dtype=np.float32)
        shape = list(xa.shape)
        d = len(shape)
        cores_np = [np.zeros((ranks[k], shape[k], ranks[k + 1]), dtype=np.float32, order="F")
                    for k in range(d)]
        ptrs = (C.c_void_p * d)(*[c.ctypes.data for c in cores_np])
        o = _opts(gemm, method, oversample, power_iters, seed, flags | TT_FLAG_HOST_IO, max_sweeps)
        o.eps = float(eps)
        torch = _torch()
        ctx = _ctx_for()
        st = _lib.TTStats()
        fn = lib().tr_svd if ring else lib().tt_svd
        check(fn(ctx, C.c_void_p(xa.ctypes.data), d, _lib.int_array(shape), _lib.int_array(ranks),
                 C.byref(o), ptrs, C.byref(st)))
        cores = cores_np
        if eps > 0:  # adaptive ranks: core k occupies the first r_k n_k r_{k+1} values of its buffer
            rr = list(st.ranks[: d + 1])
            cores = [np.asfortranarray(cores_np[k].reshape(-1, order="F")[: rr[k] * shape[k] * rr[k + 1]]
                                       .reshape(rr[k], shape[k], rr[k + 1], order="F")) for k in range(d)]
    else:
        torch = _torch()
        if shape is None:
            shape = list(x.shape)
            buf = _fortran_buffer(x)
        else:
            buf = x.reshape(-1)
        d = len(shape)
        flat = [torch.empty(ranks[k] * shape[k] * ranks[k + 1], device=buf.device, dtype=torch.float32)
                for k in range(d)]
        ptrs = (C.c_void_p * d)(*[t.data_ptr() for t in flat])
        o = _opts(gemm, method, oversample, power_iters, seed, flags, max_sweeps)
        o.eps = float(eps)
        ctx = _ctx_for(buf.device.index)
        st = _lib.TTStats()
        fn = lib().tr_svd if ring else lib().tt_svd
        check(fn(ctx, _ptr(buf), d, _lib.int_array(shape), _lib.int_array(ranks), C.byref(o), ptrs,
                 C.byref(st)))
        rr = list(st.ranks[: d + 1]) if eps > 0 else ranks
        cores = [_core_view(flat[k][: rr[k] * shape[k] * rr[k + 1]], rr[k], shape[k], rr[k + 1])
                 for k in range(d)]
    sig = [np.array(st.sigma[k][: st.nsigma[k]], dtype=np.float64) for k in range(st.nsteps)]
    ns = int(st.nsteps)
    return Result(cores=cores, ms=st.ms, sigmas=sig, ranks=list(st.ranks[: len(ranks)]),
                  kernels=st.kernels, jacobi_sweeps=st.jacobi_sweeps, est_rel_err=st.est_rel_err,
                  passes=st.passes, fallbacks=st.fallbacks, step_ks=list(st.step_ks[:ns]),
                  step_power=list(st.step_power[:ns]), step_attempts=list(st.step_attempts[:ns]),
                  eps_unmet=int(st.eps_unmet), flops=float(st.flops))


def tt_svd(x, ranks, **kw) -> Result:
    """TT-SVD of ``x`` (torch CUDA tensor or NumPy array, logical shape (n1..nd)) at fixed
    ranks ``[1, r1, ..., r_{d-1}, 1]``.  Keyword options: gemm ('auto' | 'tc' | 'fp32'),
    method ('edrsvd' | 'exact'), oversample, power_iters, seed, flags, max_sweeps, eps.
    With eps > 0 the ranks are upper bounds and every unfolding is truncated to the smallest
    rank whose discarded energy is <= eps^2 ||X||^2 / (d - 1) (TT-SVD delta-truncation);
    Result.ranks holds the ranks chosen and Result.est_rel_err the implied error bound;
    Result.eps_unmet > 0 says a rank bound (the caller's, or the 128-column sketch limit) kept the
    bound above eps (flags |= TT_FLAG_STRICT_EPS makes that an error instead).
    stream=True (NumPy input, fixed ranks): the first unfolding is streamed from host memory in
    chunks (set_stream_chunk) instead of being copied to the device whole."""
    return _run(False, x, ranks, **kw)


def tr_svd(x, ranks, **kw) -> Result:
    """TR-SVD of ``x`` with bond ranks ``[r0, r1, ..., r_{d-1}, r0]``."""
    return _run(True, x, ranks, **kw)


def rel_error(x, cores, ring: bool = False) -> float:
    """||X - TT(cores)||_F / ||X||_F on the device (FP64 accumulation)."""
    torch = _torch()
    buf = _fortran_buffer(x)
    d = x.dim()
    shape = list(x.shape)
    ranks = [cores[0].shape[0]] + [c.shape[2] for c in cores]
    flat = []
    for c in cores:
        f = c.permute(2, 1, 0).contiguous().reshape(-1)
        flat.append(f.float())
    ptrs = (C.c_void_p * d)(*[t.data_ptr() for t in flat])
    out = C.c_double()
    check(lib().tt_rel_error(_ctx_for(buf.device.index), _ptr(buf), d, _lib.int_array(shape),
                             _lib.int_array(ranks), 1 if ring else 0, ptrs, C.byref(out)))
    return float(out.value)


# ---- building blocks (torch CUDA tensors, column-major matrices as (rows, cols) tensors
#      whose memory is column-major, i.e. the transpose of a contiguous (cols, rows) tensor) ----
def _colmajor(rows, cols, dtype, device):
    torch = _torch()
    return torch.empty((cols, rows), dtype=dtype, device=device).t()


def gaussian(rows: int, cols: int, seed: int, stream_id: int = 0, device=None):
    """Column-major (rows x cols) N(0,1) matrix from the device Philox generator."""
    torch = _torch()
    out = _colmajor(rows, cols, torch.float32, device or torch.device("cuda"))
    check(lib().tt_k_gaussian(_ctx_for(out.device.index), _ptr(out), rows, cols, rows, seed, stream_id))
    return out


def _as_colmajor(a):
    """Column-major storage of a 2-D torch tensor (returns a (rows, cols) view with stride (1, rows))."""
    return a.t().contiguous().t()


def sketch(a, w, gemm="auto"):
    """Y = A W (FP64 result) with A (m x n) and W (n x N) column-major FP32."""
    torch = _torch()
    a = _as_colmajor(a.float())
    w = _as_colmajor(w.float())
    m, n = a.shape
    N = w.shape[1]
    y = _colmajor(m, N, torch.float64, a.device)
    check(lib().tt_k_sketch(_ctx_for(a.device.index), _ptr(a), m, n, _ptr(w), N, n, _ptr(y), GEMM[gemm]))
    return y


def project(a, q, gemm="auto"):
    """Q^T A as an (N x n) column-major matrix (stored row-major n x N), A (m x n), Q (m x N)."""
    torch = _torch()
    a = _as_colmajor(a.float())
    q = _as_colmajor(q.float())
    m, n = a.shape
    N = q.shape[1]
    out = torch.empty((n, N), dtype=torch.float32, device=a.device)
    check(lib().tt_k_project(_ctx_for(a.device.index), _ptr(a), m, n, _ptr(q), N, m, _ptr(out), N,
                             GEMM[gemm]))
    return out.t()


def gram_rows(a, gemm="fp32"):
    """A A^T (FP64) of a column-major (m x n) matrix, m <= 128."""
    torch = _torch()
    a = _as_colmajor(a.float())
    m, n = a.shape
    w = _colmajor(m, m, torch.float64, a.device)
    check(lib().tt_k_gram_rows(_ctx_for(a.device.index), _ptr(a), m, n, _ptr(w), GEMM[gemm]))
    return w


def gram_tall(z, rowmajor=False):
    """Z^T Z (FP64) of a tall matrix Z (n x N), column-major, or row-major (rows contiguous,
    the layout of a projected factor B^T) with rowmajor=True."""
    torch = _torch()
    if rowmajor:
        z = z.float().contiguous()
        n, N = z.shape
        rs, cs = N, 1
    else:
        z = _as_colmajor(z.float())
        n, N = z.shape
        rs, cs = 1, n
    w = _colmajor(N, N, torch.float64, z.device)
    check(lib().tt_k_gram_tall(_ctx_for(z.device.index), _ptr(z), n, N, rs, cs, _ptr(w)))
    return w


def cholqr2(y, want_r=True):
    """CholeskyQR2 of a tall matrix; returns (Q, R), or (Q, None) with want_r=False (the form the
    decomposition's sketches use: no R, which lets up to 80 columns run in one launch)."""
    torch = _torch()
    q = y.float().t().contiguous().clone().t()  # private column-major copy
    n, N = q.shape
    r = _colmajor(N, N, torch.float64, q.device) if want_r else None
    check(lib().tt_k_cholqr2(_ctx_for(q.device.index), _ptr(q), n, N, n, _ptr(r) if want_r else None))
    return q, r


def syev(w):
    """Eigen-decomposition of a symmetric FP64 matrix (descending); returns (evals, evecs, sweeps)."""
    torch = _torch()
    w = _as_colmajor(w.double())
    N = w.shape[0]
    ev = torch.empty(N, dtype=torch.float64, device=w.device)
    vec = _colmajor(N, N, torch.float64, w.device)
    sw = C.c_int()
    check(lib().tt_k_syev(_ctx_for(w.device.index), _ptr(w), N, _ptr(ev), _ptr(vec), C.byref(sw)))
    return ev, vec, sw.value


def permute231(x, r0: int, r1: int, n: int):
    """(r0, r1, n) -> (r1, n, r0) on column-major flat buffers."""
    torch = _torch()
    x = x.reshape(-1).float().contiguous()
    out = torch.empty_like(x)
    check(lib().tt_k_permute231(_ctx_for(x.device.index), _ptr(x), _ptr(out), r0, r1, n))
    return out


# ---- learned EDrSVD parameters ----
def set_predictor(params, device=None):
    """Install the predictor (TT_MLP_PARAMS floats; None clears it) in the device's context."""
    torch = _torch()
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    ctx = _ctx_for(dev.index if isinstance(dev, torch.device) else dev)
    if params is None:
        check(lib().tt_ctx_set_predictor(ctx, None))
        return
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).ravel())
    if p.size != _lib.TT_MLP_PARAMS:
        raise ValueError(f"predictor needs {_lib.TT_MLP_PARAMS} parameters, got {p.size}")
    check(lib().tt_ctx_set_predictor(ctx, C.c_void_p(p.ctypes.data)))


def probe_features(a, energy=-1.0, tol=1e-3, seed=1234, stream_id=0):
    """The TT_MLP_INPUTS probe features of a column-major (m x n) FP32 CUDA matrix."""
    torch = _torch()
    a = _as_colmajor(a.float())
    m, n = a.shape
    out = torch.empty(_lib.TT_MLP_INPUTS, dtype=torch.float32, device=a.device)
    check(lib().tt_probe_features(_ctx_for(a.device.index), _ptr(a), m, n, float(energy), float(tol), int(seed),
                                  int(stream_id), _ptr(out)))
    return out


def mlp_forward(params, x):
    """Network outputs (n x 3) for features x (n x 8), both CUDA FP32 row-major."""
    torch = _torch()
    x = x.float().contiguous()
    y = torch.empty((x.shape[0], _lib.TT_MLP_OUTPUTS), dtype=torch.float32, device=x.device)
    check(lib().tt_mlp_forward(_ctx_for(x.device.index), _ptr(params.contiguous()), _ptr(x), int(x.shape[0]), _ptr(y)))
    return y


def mlp_grad(params, x, t):
    """(gradient, loss) of the mean summed squared error over the batch."""
    torch = _torch()
    x = x.float().contiguous()
    t = t.float().contiguous()
    g = torch.empty(_lib.TT_MLP_PARAMS, dtype=torch.float32, device=x.device)
    loss = torch.empty(1, dtype=torch.float32, device=x.device)
    check(lib().tt_mlp_grad(_ctx_for(x.device.index), _ptr(params.contiguous()), _ptr(x), _ptr(t),
                            int(x.shape[0]), _ptr(g), _ptr(loss)))
    return g, loss


def mlp_train(params, adam_m, adam_v, x, t, steps, batch=256, lr=1e-3, step0=0, seed=1234):
    """Adam steps in place on CUDA tensors params / adam_m / adam_v; returns the loss trace."""
    torch = _torch()
    x = x.float().contiguous()
    t = t.float().contiguous()
    trace = torch.empty(max(int(steps), 1), dtype=torch.float32, device=x.device)
    check(lib().tt_mlp_train(_ctx_for(x.device.index), _ptr(params), _ptr(adam_m), _ptr(adam_v), _ptr(x), _ptr(t),
                             int(x.shape[0]), int(steps), int(batch), float(lr), int(step0), int(seed), _ptr(trace)))
    return trace[: int(steps)]


# ---- batched small tensors ----
class Batch:
    """A packed batch of small tensors for ``tt_svd_batched``: the column-major tensors in one
    device buffer, their offsets, and the room for their cores."""

    def __init__(self, tensors, rmax=16, device=None):
        torch = _torch()
        self.device = device or torch.device("cuda")
        self.shapes = [list(t.shape) for t in tensors]
        self.d = len(self.shapes[0])
        if any(len(sh) != self.d for sh in self.shapes):
            raise ValueError("all tensors need the same order")
        self.rmax = int(rmax)
        sizes = [int(np.prod(sh)) for sh in self.shapes]
        self.x_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.flat = torch.empty(int(sum(sizes)), dtype=torch.float32, device=self.device)
        for t, off, sz in zip(tensors, self.x_off, sizes):
            if isinstance(t, np.ndarray):
                src = torch.from_numpy(np.ascontiguousarray(np.asarray(t, dtype=np.float32).ravel(order="F")))
            else:
                src = t.permute(*reversed(range(t.dim()))).reshape(-1).float()
            self.flat[int(off):int(off) + sz] = src.to(self.device)
        caps = [int(lib().tt_batch_core_capacity(self.d, _lib.int_array(sh), self.rmax)) for sh in self.shapes]
        self.core_off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
        self.cores = torch.zeros(int(sum(caps)), dtype=torch.float32, device=self.device)
        self.count = len(tensors)
        self.n_arr = (C.c_int * (self.count * self.d))(*[int(v) for sh in self.shapes for v in sh])
        self.ranks = (C.c_int * (self.count * (self.d + 1)))()
        self.err = (C.c_double * self.count)()
        self.plan = None
        self.plan_args = None

    def make_plan(self, eps=1e-2, oversample=8, seed=20261203):
        """Create the batch plan (shape table, work orders and scratch kept on the device)."""
        self.close()
        ctx = _ctx_for(self.device.index)
        p = C.c_void_p()
        check(lib().tt_batch_plan_create(ctx, self.count, self.d, self.n_arr,
                                         self.x_off.ctypes.data_as(C.POINTER(C.c_longlong)), float(eps), self.rmax,
                                         int(oversample), int(seed),
                                         self.core_off.ctypes.data_as(C.POINTER(C.c_longlong)), C.byref(p)))
        self.plan = p
        self.plan_args = (float(eps), int(oversample), int(seed))

    def tune(self, reps=2):
        """Time every kernel variant on this batch and keep the fastest; returns the 6 times
        (ms; chunk 16/32/64 in natural order, then largest-first)."""
        if self.plan is None:
            self.make_plan()
        ms = (C.c_float * 6)()
        check(lib().tt_batch_plan_tune(self.plan, C.c_void_p(self.flat.data_ptr()), C.c_void_p(self.cores.data_ptr()),
                                       int(reps), ms))
        return list(ms)

    def variant(self):
        """(sketch chunk width, largest-first work order) of the plan."""
        ch, lf = C.c_int(), C.c_int()
        check(lib().tt_batch_plan_variant(self.plan, C.byref(ch), C.byref(lf)))
        return ch.value, bool(lf.value)

    def run(self, eps=1e-2, oversample=8, seed=20261203, graph=True):
        """Decompose the packed tensors (results stay in the Batch).  graph=True replays the
        plan's CUDA graph (created on first use); graph=False makes one tt_svd_batched call."""
        if graph:
            if self.plan is None or self.plan_args != (float(eps), int(oversample), int(seed)):
                self.make_plan(eps, oversample, seed)
            check(lib().tt_batch_plan_run(self.plan, C.c_void_p(self.flat.data_ptr()),
                                          C.c_void_p(self.cores.data_ptr()), self.ranks, self.err))
            return
        ctx = _ctx_for(self.device.index)
        check(lib().tt_svd_batched(ctx, self.count, self.d, self.n_arr, C.c_void_p(self.flat.data_ptr()),
                                   self.x_off.ctypes.data_as(C.POINTER(C.c_longlong)), float(eps), self.rmax,
                                   int(oversample), int(seed), C.c_void_p(self.cores.data_ptr()),
                                   self.core_off.ctypes.data_as(C.POINTER(C.c_longlong)), self.ranks, self.err))

    def close(self):
        if getattr(self, "plan", None) is not None:
            lib().tt_batch_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def results(self):
        """Per tensor: (cores as CUDA tensors of logical shape (r_k, n_k, r_{k+1}), ranks, err_est)."""
        d = self.d
        out = []
        for t in range(self.count):
            rr = [self.ranks[t * (d + 1) + k] for k in range(d + 1)]
            off = int(self.core_off[t])
            cs = []
            for k in range(d):
                cnt = rr[k] * self.shapes[t][k] * rr[k + 1]
                cs.append(_core_view(self.cores[off:off + cnt], rr[k], self.shapes[t][k], rr[k + 1]))
                off += cnt
            out.append((cs, rr, self.err[t]))
        return out


def tt_svd_batched(tensors, eps=1e-2, rmax=16, oversample=8, seed=20261203, device=None):
    """TT-SVD of many small tensors in one persistent launch (``tt_svd_batched``).

    ``tensors``: list of NumPy arrays (same order d, any mode sizes) or of CUDA tensors with
    their logical shapes.  Returns a list of (cores, ranks, err_est) per tensor; cores are CUDA
    tensors with logical shape (r_k, n_k, r_{k+1})."""
    b = Batch(tensors, rmax=rmax, device=device)
    b.run(eps=eps, oversample=oversample, seed=seed, graph=False)
    return b.results()


# ---- core files ----
def save_cores(path: str, cores, ring: bool = False) -> None:
    """Write cores (logical (r_{k-1}, n_k, r_k) arrays, NumPy or torch, host or CUDA) to a
    core file (format in include/ttrsvd.h)."""
    d = len(cores)
    n = [int(c.shape[1]) for c in cores]
    r = [int(cores[0].shape[0])] + [int(c.shape[2]) for c in cores]
    host = []
    for c in cores:
        if hasattr(c, "detach"):
            c = c.detach().float().cpu().numpy()
        host.append(np.asfortranarray(np.asarray(c, dtype=np.float32)))
    ptrs = (C.c_void_p * d)(*[h.ctypes.data for h in host])
    check(lib().tt_cores_save(os.fsencode(path), d, _lib.int_array(n), _lib.int_array(r), 1 if ring else 0,
                              ptrs, 0))


def load_cores(path: str):
    """Read a core file; returns (cores as column-major NumPy arrays, ring)."""
    d = C.c_int()
    ring = C.c_int()
    n = (C.c_int * _lib.TT_MAX_ORDER)()
    r = (C.c_int * (_lib.TT_MAX_ORDER + 1))()
    check(lib().tt_cores_header(os.fsencode(path), C.byref(d), n, r, C.byref(ring)))
    cores = [np.empty((r[k], n[k], r[k + 1]), dtype=np.float32, order="F") for k in range(d.value)]
    ptrs = (C.c_void_p * d.value)(*[c.ctypes.data for c in cores])
    check(lib().tt_cores_load(os.fsencode(path), ptrs, 0))
    return cores, bool(ring.value)


# ---- reference-compatible entry points (host NumPy tensors, column-major) ----
def _host_f32(h):
    a = np.asarray(h)
    if a.dtype != np.float32 or not (a.flags.f_contiguous or a.ndim == 1):
        a = np.asfortranarray(a, dtype=np.float32)
    return a


def ttdec_gpu_float(h_tensor, h_n_array, h_r_array, eps=None, single_error=None, single_com_ratio=None):
    """Order-3 TT-SVD; mirrors ttdec_gpu_float (ttdec_gpu_float_rsvd_lu_half.cu:778).
    Returns elapsed seconds.  ``single_error``/``single_com_ratio``: optional 1-element float32
    arrays that receive ||X-X^||/||X|| and the compression ratio."""
    a = _host_f32(h_tensor)
    e = np.zeros(1, np.float32) if single_error is None else single_error
    cr = np.zeros(1, np.float32) if single_com_ratio is None else single_com_ratio
    t = lib().tt_ref_ttdec_gpu_float(
        C.c_void_p(a.ctypes.data), _lib.int_array(h_n_array), _lib.int_array(h_r_array), None,
        e.ctypes.data_as(C.POINTER(C.c_float)) if single_error is not None else None,
        cr.ctypes.data_as(C.POINTER(C.c_float)) if single_com_ratio is not None else None)
    if t < 0:
        raise TTError(int(-t), lib().tt_last_error().decode())
    return float(t)


def trdec_gpu_float(h_tensor, h_n_array, h_r_array, eps=None, single_error=None, single_com_ratio=None):
    """Order-3 TR-SVD; mirrors trdec_gpu_float (trdec_gpu_float_rsvd_lu_half.cu:734)."""
    a = _host_f32(h_tensor)
    t = lib().tt_ref_trdec_gpu_float(
        C.c_void_p(a.ctypes.data), _lib.int_array(h_n_array), _lib.int_array(h_r_array), None,
        single_error.ctypes.data_as(C.POINTER(C.c_float)) if single_error is not None else None,
        single_com_ratio.ctypes.data_as(C.POINTER(C.c_float)) if single_com_ratio is not None else None)
    if t < 0:
        raise TTError(int(-t), lib().tt_last_error().decode())
    return float(t)


def ttdec_half_lu_device_6(h_A, ttRanks, ttDemns, calculateTimes=1, p=64, calError=False):
    """Order-6 TT-SVD; mirrors ttdec_half_lu_device_6 (ttdec6_singleGPU.cu:799)."""
    a = _host_f32(h_A)
    t = lib().tt_ref_ttdec_half_lu_device_6(C.c_void_p(a.ctypes.data), _lib.int_array(ttRanks),
                                            _lib.int_array(ttDemns), int(calculateTimes), int(p),
                                            1 if calError else 0)
    if t < 0:
        raise TTError(int(-t), lib().tt_last_error().decode())
    return float(t)


def ttdec_half_lu_host_6(h_A, ttRanks, ttDemns, calculateTimes=1, p=8, calError=False):
    """Order-6 TT-SVD with the tensor left in host memory and its first unfolding streamed in
    p slices; mirrors ttdec_half_lu_host_6 (ttdec6_singleGPU.cu:656)."""
    a = _host_f32(h_A)
    t = lib().tt_ref_ttdec_half_lu_host_6(C.c_void_p(a.ctypes.data), _lib.int_array(ttRanks),
                                          _lib.int_array(ttDemns), int(calculateTimes), int(p),
                                          1 if calError else 0)
    if t < 0:
        raise TTError(int(-t), lib().tt_last_error().decode())
    return float(t)


def trdec_half_lu_device_6(h_A, ttRanks, ttDemns, calculateTimes=1, p=64, calError=False):
    """Order-6 TR-SVD; mirrors the TR ttdec_half_lu_device_6 (trdec6_singleGPU.cu:827)."""
    a = _host_f32(h_A)
    t = lib().tt_ref_trdec_half_lu_device_6(C.c_void_p(a.ctypes.data), _lib.int_array(ttRanks),
                                            _lib.int_array(ttDemns), int(calculateTimes), int(p),
                                            1 if calError else 0)
    if t < 0:
        raise TTError(int(-t), lib().tt_last_error().decode())
    return float(t)
