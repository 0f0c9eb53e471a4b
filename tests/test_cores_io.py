"""Core file format (tt_cores_save / tt_cores_header / tt_cores_load): host-side, no GPU."""
import os
import struct

import numpy as np
import pytest

import oracle


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


@pytest.mark.parametrize("ring", [False, True])
def test_roundtrip_oracle_cores(tmp_path, ring):
    ttr = _ttr()
    rng = np.random.default_rng(3)
    shape = [4, 5, 3, 6]
    if ring:
        cores = oracle.tr_random_cores(shape, 3, rng, dtype=np.float32)
    else:
        cores = oracle.tt_random_cores(shape, [1, 2, 4, 3, 1], rng, dtype=np.float32)
    path = str(tmp_path / "x.ttr")
    ttr.save_cores(path, cores, ring=ring)
    back, ring_back = ttr.load_cores(path)
    assert ring_back == ring
    assert [c.shape for c in back] == [c.shape for c in cores]
    for a, b in zip(cores, back):
        assert np.array_equal(np.asarray(a, dtype=np.float32), b)
    full = oracle.tr_full(back) if ring else oracle.tt_full(back)
    ref = oracle.tr_full(cores) if ring else oracle.tt_full(cores)
    np.testing.assert_allclose(full, ref, rtol=1e-6, atol=1e-6)


def test_layout_is_documented_header(tmp_path):
    ttr = _ttr()
    cores = [np.arange(6, dtype=np.float32).reshape(1, 2, 3, order="F"),
             np.arange(12, dtype=np.float32).reshape(3, 4, 1, order="F")]
    path = str(tmp_path / "h.ttr")
    ttr.save_cores(path, cores)
    raw = open(path, "rb").read()
    assert raw[:8] == b"TTRCORE1"
    kind, d, dtype, _ = struct.unpack("<4i", raw[8:24])
    assert (kind, d, dtype) == (0, 2, 0)
    n = struct.unpack("<2q", raw[24:40])
    r = struct.unpack("<3q", raw[40:64])
    assert n == (2, 4) and r == (1, 3, 1)
    data = np.frombuffer(raw[64:], dtype="<f4")
    assert np.array_equal(data[:6], cores[0].ravel(order="F"))
    assert np.array_equal(data[6:], cores[1].ravel(order="F"))


def test_bad_files_raise_io_error(tmp_path):
    ttr = _ttr()
    from tensor_train_ring_decompositions_hpc_gpu_b200._lib import TTError
    bad = tmp_path / "bad.ttr"
    bad.write_bytes(b"NOTACORE" + b"\0" * 64)
    with pytest.raises(TTError) as e:
        ttr.load_cores(str(bad))
    assert e.value.code == 10
    with pytest.raises(TTError) as e:
        ttr.load_cores(str(tmp_path / "missing.ttr"))
    assert e.value.code == 10
    cores = [np.ones((1, 3, 2), dtype=np.float32), np.ones((2, 3, 1), dtype=np.float32)]
    good = str(tmp_path / "t.ttr")
    ttr.save_cores(good, cores)
    raw = open(good, "rb").read()
    trunc = tmp_path / "trunc.ttr"
    trunc.write_bytes(raw[:-4])
    with pytest.raises(TTError) as e:
        ttr.load_cores(str(trunc))
    assert e.value.code == 10
