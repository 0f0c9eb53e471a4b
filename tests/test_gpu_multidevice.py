"""Two devices in one process: kernel attributes, SM counts and the static scratch address are
per device, so the large-shared-memory kernels and the allocation-free sketch run on device 1
after device 0 has been used.  Skipped unless two GPUs are visible."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cm(rows, cols, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn((cols, rows), generator=g, dtype=torch.float32).to(dev).t()


@pytest.fixture(scope="module")
def two_gpus(gpu):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    return [torch.device("cuda:0"), torch.device("cuda:1")]


@pytest.mark.parametrize("gemm", ["tc", "fp32"])
def test_sketch_on_two_devices(two_gpus, gemm):
    import torch
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    lib = ttr.lib()
    m, n, N = 1024, 120000, 40
    for dev in two_gpus:
        with torch.cuda.device(dev):
            a = _cm(m, n, 5, dev)
            w = _cm(n, N, 6, dev)
            ref = a.double().cpu().numpy() @ w.double().cpu().numpy()
            y1 = ttr.sketch(a, w, gemm).cpu().numpy()
            y2 = torch.empty((N, m), dtype=torch.float64, device=dev).t()
            stream = torch.cuda.current_stream(dev).cuda_stream
            torch.cuda.synchronize(dev)
            rc = lib.tt_k_sketch_noalloc(C.c_void_p(a.data_ptr()), m, n, C.c_void_p(w.data_ptr()), N, n,
                                         C.c_void_p(y2.data_ptr()), ttr.GEMM[gemm], C.c_void_p(stream))
            assert rc == 0, lib.tt_last_error()
            tol = 3e-3 if gemm == "tc" else 2e-6
            for y in (y1, y2.cpu().numpy()):
                assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < tol


def test_noalloc_rejects_stream_of_other_device(two_gpus):
    import torch
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    lib = ttr.lib()
    with torch.cuda.device(two_gpus[1]):
        s1 = torch.cuda.Stream(two_gpus[1])
    with torch.cuda.device(two_gpus[0]):
        rc = lib.tt_k_sketch_noalloc(C.c_void_p(256), 64, 64, C.c_void_p(256), 8, 64, C.c_void_p(256), 0,
                                     C.c_void_p(s1.cuda_stream))
    assert rc == 1 and b"stream belongs to device" in lib.tt_last_error()
