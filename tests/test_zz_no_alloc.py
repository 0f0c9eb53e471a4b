"""tt_k_sketch_noalloc: the allocation-free sketch entry point (static device scratch).

It serves callers that must not call cudaMalloc (device memory owned by another allocator
or a pre-reserved arena, or loops that cannot afford cudaMalloc's device synchronisation).
Checked through the C ABI against the context-based tt_k_sketch on two calls in a row, since
every call reuses the same static scratch array.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cm(rows, cols, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn((cols, rows), generator=g, dtype=torch.float32).to(dev).t()


@pytest.mark.parametrize("gemm", ["tc", "fp32"])
def test_noalloc_sketch_matches_context_sketch_twice(gpu, gemm):
    import torch
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = ttr.lib()
    stream = torch.cuda.current_stream(gpu).cuda_stream
    for call, (m, n, N) in enumerate([(1024, 200000, 40), (256, 77777, 24)]):
        a = _cm(m, n, 11 + call, gpu)
        w = _cm(n, N, 21 + call, gpu)
        ref = ttr.sketch(a, w, gemm)  # the existing entry point (context workspace)
        y = torch.empty((N, m), dtype=torch.float64, device=gpu).t()
        torch.cuda.synchronize(gpu)
        rc = lib.tt_k_sketch_noalloc(C.c_void_p(a.data_ptr()), m, n, C.c_void_p(w.data_ptr()), N, n,
                                     C.c_void_p(y.data_ptr()), ttr.GEMM[gemm], C.c_void_p(stream))
        assert rc == 0, lib.tt_last_error()
        got = y.cpu().numpy()
        exp = ref.cpu().numpy()
        # same kernel; only the number of column splits (summation order) may differ
        rel = np.linalg.norm(got - exp) / np.linalg.norm(exp)
        assert rel < 1e-5, (call, rel)


def test_noalloc_rejects_oversized_partials(gpu):
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    lib = ttr.lib()
    m, N = 1 << 16, 64  # m * N = 2^22 doubles > the 2^21-double scratch
    rc = lib.tt_k_sketch_noalloc(C.c_void_p(16), m, 1024, C.c_void_p(16), N, 1024, C.c_void_p(16), 0, None)
    assert rc == 2 and b"static scratch" in lib.tt_last_error()
