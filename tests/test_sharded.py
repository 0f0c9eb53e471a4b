"""Column-sharded TT-SVD (sharded.tt_svd_sharded): the orchestration on CPU ranks over gloo with
a NumPy backend, and the CUDA backend on one GPU as a one-rank NCCL group."""
import os
import socket

import numpy as np
import pytest

import oracle
from tensor_train_ring_decompositions_hpc_gpu_b200 import sharded


class Arr:
    """An array of the NumPy test backend that refuses host arithmetic: NumPy functions,
    ufuncs and operators on it raise, so every computation of the sharded chain must go through
    a backend method (as it does on the device backend)."""
    __slots__ = ("v",)
    __array_ufunc__ = None

    def __init__(self, v):
        self.v = np.asarray(v, dtype=np.float64)

    def __array__(self, *args, **kwargs):
        raise TypeError("host arithmetic on a backend array")


def _v(a):
    return a.v if isinstance(a, Arr) else np.asarray(a, dtype=np.float64)


class NumpyBackend:
    """The operations of ``sharded.DeviceBackend`` in FP64 NumPy (column-major matrices), on
    opaque arrays."""

    def matrix(self, flat, rows, cols):
        return Arr(_v(flat)[: rows * cols].reshape(rows, cols, order="F"))

    def flat(self, a):
        return Arr(_v(a).ravel(order="F"))

    def cols(self, a, c0, c1):
        return Arr(_v(a)[:, c0:c1])

    def vcat(self, blocks):
        return Arr(np.vstack([_v(b) for b in blocks]))

    def pad_cols(self, a, n):
        x = _v(a)
        out = np.zeros((x.shape[0], max(n, x.shape[1])))
        out[:, : x.shape[1]] = x
        return Arr(out)

    def permute231(self, flat, r0, r1, n):
        return Arr(_v(flat).reshape(r0, r1, n, order="F").transpose(1, 2, 0).ravel(order="F"))

    def gram_rows(self, a):
        x = _v(a)
        return Arr(x @ x.T)

    def gram_cols(self, a):
        x = _v(a)
        return Arr(x.T @ x)

    def sketch(self, a, w):
        return Arr(_v(a) @ _v(w))

    def project(self, a, q):
        return Arr(_v(q).T @ _v(a))

    def omega_rows(self, row0, nrows, total_rows, cols, seed, stream):
        return Arr(oracle.gaussian_from_philox(total_rows, cols, seed, stream)[row0:row0 + nrows])

    def cholqr(self, y):
        q, r = np.linalg.qr(_v(y))
        return Arr(q * np.where(np.diag(r) < 0, -1.0, 1.0))

    def syev(self, w):
        x = _v(w)
        lam, v = np.linalg.eigh(0.5 * (x + x.T))
        return Arr(lam[::-1]), Arr(v[:, ::-1])

    def inv_sqrt_psd(self, w, rel_floor=1e-12):
        lam, v = self.syev(w)
        lam, v = _v(lam), _v(v)
        keep = lam > rel_floor * max(lam[0], 1e-300)
        s = np.where(keep, 1.0 / np.sqrt(np.maximum(lam, 1e-300)), 0.0)
        return Arr((v * s) @ v.T)

    def canon(self, u):
        x = _v(u)
        idx = np.argmax(np.abs(x), axis=0)
        sg = np.where(x[idx, np.arange(x.shape[1])] < 0, -1.0, 1.0)
        return Arr(x * sg), Arr(sg)

    def scale_cols(self, a, s):
        return Arr(_v(a) * _v(s)[None, :])

    def scale_rows(self, a, s):
        return Arr(_v(a) * _v(s)[:, None])

    def sigma(self, ev, r):
        return Arr(np.sqrt(np.maximum(_v(ev)[:r], 0.0)))

    def recip(self, s):
        x = _v(s)
        return Arr(np.where(x > 0, 1.0 / np.where(x > 0, x, 1.0), 0.0))

    def head(self, v, r):
        return Arr(_v(v)[:, :r])

    def t(self, a):
        return Arr(_v(a).T)

    def to_host(self, t):
        return np.array(_v(t), dtype=np.float64)

    def allreduce(self, t, group):
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            return t
        tt = torch.from_numpy(np.ascontiguousarray(_v(t)))
        dist.all_reduce(tt, group=group)
        return Arr(tt.numpy())

    def allgather_cols(self, a, group):
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            return a
        world = dist.get_world_size(group)
        mine = torch.from_numpy(np.ascontiguousarray(_v(a).T))
        blocks = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(blocks, mine, group=group)
        return Arr(torch.cat(blocks, dim=0).numpy().T)


SHAPE = [12, 12, 10, 8, 16]
RANKS = [1, 10, 10, 8, 6, 1]
# ring with bond 2: step 1 exact (rank r0 r1 = 4 of 10 rows), step 2 sketched (80 rows),
# steps 3 and 4 exact
TR_SHAPE = [10, 40, 6, 6, 8]
TR_RANKS = [2, 2, 2, 2, 2, 2]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_block(x, world, rank):
    nloc = x.shape[-1] // world
    return np.asfortranarray(x[..., rank * nloc:(rank + 1) * nloc]).ravel(order="F").astype(np.float64)


def _worker(rank, world, port, x, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cores, used = sharded.tt_svd_sharded(Arr(_local_block(x, world, rank)), list(x.shape), RANKS,
                                             oversample=6, power_iters=1, seed=77, backend=NumpyBackend())
        np.savez(os.path.join(out_dir, f"w{world}_r{rank}.npz"), *cores, used=np.array(used))
        xr = oracle.make_tr_tensor(TR_SHAPE, 2, 1e-6, seed=43).astype(np.float64)
        cores, used = sharded.tr_svd_sharded(Arr(_local_block(xr, world, rank)), TR_SHAPE, TR_RANKS,
                                             oversample=6, power_iters=1, seed=79, backend=NumpyBackend())
        np.savez(os.path.join(out_dir, f"tr_w{world}_r{rank}.npz"), *cores, used=np.array(used))
    finally:
        dist.destroy_process_group()


def _run(world, x, out_dir):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), x, out_dir), nprocs=world, join=True)
    res, tr = [], []
    for r in range(world):
        f = np.load(os.path.join(out_dir, f"w{world}_r{r}.npz"))
        res.append(([f[f"arr_{k}"] for k in range(len(SHAPE))], list(f["used"])))
        f = np.load(os.path.join(out_dir, f"tr_w{world}_r{r}.npz"))
        tr.append(([f[f"arr_{k}"] for k in range(len(TR_SHAPE))], list(f["used"])))
    return res, tr


@pytest.fixture(scope="module")
def sharded_runs(tmp_path_factory):
    x = oracle.make_tt_tensor(SHAPE, RANKS, 1e-6, seed=41).astype(np.float64)
    d = str(tmp_path_factory.mktemp("sharded"))
    (one, tr1), (two, tr2) = _run(1, x, d), _run(2, x, d)
    return x, one, two, tr1, tr2


def test_sharded_ranks_agree_and_match_one_rank(sharded_runs):
    """Both ranks end with the same cores, and two ranks reproduce the one-rank chain: the
    all-reduced Grams and sketches equal the unsharded ones up to summation order, and each
    rank draws exactly its rows of the one Gaussian test matrix."""
    x, one, two, _, _ = sharded_runs
    (c1, u1), = one
    (ca, ua), (cb, ub) = two
    assert u1 == ua == ub == RANKS
    for a, b, c in zip(ca, cb, c1):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_allclose(a, c, rtol=0, atol=1e-9 * np.abs(c).max())


def test_sharded_reconstruction_matches_exact_chain(sharded_runs):
    """The sharded chain (exact steps where the small side is <= 64, sketched ones otherwise,
    an all-gather step where the columns are few) reconstructs the tensor as well as the
    oracle's exact Gram-eigen chain."""
    x, one, two, _, _ = sharded_runs
    ocores, _ = oracle.tt_svd(x, RANKS, method="gram")
    oerr = oracle.rel_error(x, oracle.tt_full(ocores))
    err = oracle.rel_error(x, oracle.tt_full(two[0][0]))
    assert abs(err - oerr) < 1e-6, (err, oerr)


def test_sharded_ring_ranks_agree_and_match_exact_chain(sharded_runs):
    """TR-SVD with the last mode split over two ranks (r0 strided column blocks after the 231
    permute): both ranks agree, two ranks reproduce one, and the reconstruction matches the
    oracle's exact TR chain."""
    _, _, _, tr1, tr2 = sharded_runs
    xr = oracle.make_tr_tensor(TR_SHAPE, 2, 1e-6, seed=43).astype(np.float64)
    (c1, u1), = tr1
    (ca, ua), (cb, ub) = tr2
    assert u1 == ua == ub == TR_RANKS
    for a, b, c in zip(ca, cb, c1):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_allclose(a, c, rtol=0, atol=1e-9 * np.abs(c).max())
    ocores, _ = oracle.tr_svd(xr, TR_RANKS, method="gram")
    oerr = oracle.rel_error(xr, oracle.tr_full(ocores))
    err = oracle.rel_error(xr, oracle.tr_full(ca))
    assert abs(err - oerr) < 1e-6, (err, oerr)


def test_sharded_chain_does_no_host_arithmetic():
    """The test backend's arrays refuse NumPy functions, ufuncs and operators; a chain that
    factorised anything on the host instead of through the backend would raise here."""
    with pytest.raises(TypeError):
        np.linalg.cholesky(Arr(np.eye(3)))
    with pytest.raises(TypeError):
        _ = Arr(np.eye(2)) @ Arr(np.eye(2))
    x = oracle.make_tt_tensor([6, 5, 4, 6], [1, 3, 3, 2, 1], 1e-6, seed=3).astype(np.float64)
    cores, used = sharded.tt_svd_sharded(Arr(np.asfortranarray(x).ravel(order="F")), [6, 5, 4, 6],
                                         [1, 3, 3, 2, 1], backend=NumpyBackend())
    assert used == [1, 3, 3, 2, 1]
    assert oracle.rel_error(x, oracle.tt_full(cores)) < 1e-5


def test_sharded_rejects_uneven_split():
    import torch.distributed as dist
    assert not dist.is_initialized()
    with pytest.raises(ValueError):
        # the split is checked before any collective: a one-rank view of a 3-way split
        orig = (dist.is_initialized, dist.get_world_size, dist.get_rank)
        dist.is_initialized = lambda: True
        dist.get_world_size = lambda group=None: 3
        dist.get_rank = lambda group=None: 0
        try:
            sharded.tt_svd_sharded(np.zeros(8 * 4), [8, 4], [1, 4, 1], backend=NumpyBackend())
        finally:
            dist.is_initialized, dist.get_world_size, dist.get_rank = orig


@pytest.mark.gpu
def test_sharded_device_backend_one_rank_matches_library(gpu):
    """The CUDA backend as a one-rank NCCL group: its cores reconstruct the tensor like the
    single-GPU library chain (same plan rule, same Gaussian test matrix)."""
    import datetime
    import torch
    import torch.distributed as dist
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    x = oracle.make_tt_tensor(SHAPE, RANKS, 1e-6, seed=41)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        flat = torch.from_numpy(np.asfortranarray(x).ravel(order="F")).to(gpu)
        cores, used = sharded.tt_svd_sharded(flat, SHAPE, RANKS, oversample=6, power_iters=1, seed=77,
                                             backend=sharded.DeviceBackend(gpu, gemm="fp32"))
    finally:
        dist.destroy_process_group()
    assert used == RANKS
    err = oracle.rel_error(x, oracle.tt_full(cores))
    res = ttr.tt_svd(x, RANKS, gemm="fp32")
    lerr = oracle.rel_error(x, oracle.tt_full([np.asarray(c, dtype=np.float64) for c in res.cores]))
    assert abs(err - lerr) < 1e-5, (err, lerr)


@pytest.mark.gpu
def test_sharded_ring_device_backend_one_rank(gpu):
    """TR-SVD through the CUDA backend as a one-rank NCCL group: every factorisation on the GPU,
    reconstruction as the oracle's exact TR chain."""
    import datetime
    import torch
    import torch.distributed as dist
    xr = oracle.make_tr_tensor(TR_SHAPE, 2, 1e-6, seed=43)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        flat = torch.from_numpy(np.asfortranarray(xr).ravel(order="F")).to(gpu)
        cores, used = sharded.tr_svd_sharded(flat, TR_SHAPE, TR_RANKS, oversample=6, power_iters=1, seed=79,
                                             backend=sharded.DeviceBackend(gpu, gemm="fp32"))
    finally:
        dist.destroy_process_group()
    assert used == TR_RANKS
    ocores, _ = oracle.tr_svd(xr.astype(np.float64), TR_RANKS, method="gram")
    oerr = oracle.rel_error(xr, oracle.tr_full(ocores))
    err = oracle.rel_error(xr, oracle.tr_full(cores))
    assert abs(err - oerr) < 1e-4, (err, oerr)
