"""The C ABI library: builds, loads without a GPU and exports every symbol of include/ttrsvd.h."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    src = open(os.path.join(ROOT, "include", "ttrsvd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", src)
    skip = {"sizeof", "if", "defined"}
    return sorted({n for n in names if n.startswith(("tt_", "tr_")) and n not in skip})


def test_header_declarations_exported():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = _lib.load()
    names = _header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(set(_lib.EXPORTED)) == names


def test_reference_cpp_symbols_exported():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    import subprocess
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    for sig in ["ttdec_gpu_float(float*, int*, int*, double*, float*, float*)",
                "trdec_gpu_float(float*, int*, int*, double*, float*, float*)",
                "ttdec_half_lu_device_6(float*, int const*, int const*, int const&, int const&, bool)",
                "trdec_half_lu_device_6(float*, int const*, int const*, int const&, int const&, bool)",
                "ttdec_half_lu_host_6(float*, int*, int const*, int const&, int const&, bool)"]:
        assert sig in out, sig


def test_abi_version_and_defaults():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = _lib.load()
    assert lib.tt_abi_version() == 4
    o = _lib.TTOpts()
    lib.tt_default_opts(C.byref(o))
    assert o.oversample == 8 and o.gemm == 0 and o.max_sweeps == 40


def test_null_arguments_rejected_without_gpu():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = _lib.load()
    n = _lib.int_array([4, 4, 4])
    r = _lib.int_array([1, 2, 2, 1])
    assert lib.tt_svd(None, None, 3, n, r, None, None, None) == 1  # TT_ERR_ARG
    assert lib.tr_svd(None, None, 3, n, r, None, None, None) == 1
    assert b"null" in lib.tt_last_error()
    assert lib.tt_ctx_create(None, 0, None) == 1


def test_ctx_create_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = _lib.load()
    p = C.c_void_p()
    st = lib.tt_ctx_create(C.byref(p), 0, None)
    assert st != 0 and not p.value


def test_noalloc_rejects_bad_gemm_option_without_gpu():
    """An unknown gemm value is an argument error, checked before any device work."""
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    lib = _lib.load()
    fake = C.c_void_p(256)  # never dereferenced: the option check comes first
    for bad in (-1, 3, 7):
        assert lib.tt_k_sketch_noalloc(fake, 64, 64, fake, 8, 64, fake, bad, None) == 1  # TT_ERR_ARG
        assert b"gemm option" in lib.tt_last_error()
