"""Failure handling without a GPU fault: an allocation failure injected on the host side of the
context (TT_ERR_NOMEM, the context stays usable), and a bounded device wait that runs out
(TT_ERR_TIMEOUT read from the status word, the context stays usable)."""
import time

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


def _small_tensor(gpu, seed=3):
    import torch
    x = oracle.make_tt_tensor([16, 16, 16, 16], [1, 4, 4, 4, 1], 1e-4, seed=seed)
    return torch.from_numpy(np.asfortranarray(x, dtype=np.float32)).to(gpu), x


def test_injected_allocation_failure(gpu):
    ttr = _ttr()
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = ttr.lib()
    # a fresh context on another stream, so the shared context's workspace is not already large
    import torch
    import ctypes as C
    stream = torch.cuda.Stream(gpu)
    ctx = C.c_void_p()
    assert lib.tt_ctx_create(C.byref(ctx), gpu.index or 0, C.c_void_p(stream.cuda_stream)) == 0
    try:
        xd, x = _small_tensor(gpu)
        n, r = [16] * 4, [1, 4, 4, 4, 1]
        cores = [torch.empty(r[k] * n[k] * r[k + 1], device=gpu) for k in range(4)]
        ptrs = (C.c_void_p * 4)(*[t.data_ptr() for t in cores])
        o = ttr._opts("auto", "edrsvd", 8, 0, 1, 0, 40)
        assert lib.tt_ctx_set_alloc_limit(ctx, 4096) == 0
        rc = lib.tt_svd(ctx, C.c_void_p(xd.data_ptr()), 4, _lib.int_array(n), _lib.int_array(r), C.byref(o), ptrs,
                        None)
        assert rc == 5 and b"allocation limit" in lib.tt_last_error()  # TT_ERR_NOMEM
        assert lib.tt_ctx_set_alloc_limit(ctx, 0) == 0
        rc = lib.tt_svd(ctx, C.c_void_p(xd.data_ptr()), 4, _lib.int_array(n), _lib.int_array(r), C.byref(o), ptrs,
                        None)
        assert rc == 0, lib.tt_last_error()
        torch.cuda.synchronize(gpu)
        g = [ttr._core_view(cores[k], r[k], n[k], r[k + 1]).double().cpu().numpy() for k in range(4)]
        assert oracle.rel_error(x, oracle.tt_full(g)) < 1e-3
    finally:
        lib.tt_ctx_destroy(ctx)


def test_wait_limit_runs_out_and_context_survives(gpu):
    ttr = _ttr()
    lib = ttr.lib()
    ctx = ttr._ctx_for(gpu.index or 0)
    assert lib.tt_ctx_set_wait_limit(ctx, 5_000_000) == 0  # 5 ms
    try:
        t0 = time.time()
        rc = lib.tt_k_wait_selftest(ctx)
        dt = time.time() - t0
        assert rc == 7 and b"device status 7" in lib.tt_last_error()  # TT_ERR_TIMEOUT
        assert dt < 1.0
    finally:
        assert lib.tt_ctx_set_wait_limit(ctx, 0) == 0
    # the context and the device stay usable
    xd, x = _small_tensor(gpu, seed=5)
    res = ttr.tt_svd(xd, [1, 4, 4, 4, 1])
    g = [c.double().cpu().numpy() for c in res.cores]
    assert oracle.rel_error(x, oracle.tt_full(g)) < 1e-3
