"""Column-sharded TT-SVD (sharded.tt_svd_sharded): the orchestration on CPU ranks over gloo with
a NumPy backend, and the CUDA backend on one GPU as a one-rank NCCL group."""
import os
import socket

import numpy as np
import pytest

import oracle
from tensor_train_ring_decompositions_hpc_gpu_b200 import sharded


class NumpyBackend:
    """The bulk operations of ``sharded.DeviceBackend`` in FP64 NumPy (column-major matrices)."""

    def matrix(self, flat, rows, cols):
        return np.asarray(flat[: rows * cols]).reshape(rows, cols, order="F")

    def flat(self, a):
        return np.asarray(a).ravel(order="F")

    def transpose(self, a):
        return a.T

    def gram_rows(self, a):
        return a @ a.T

    def sketch(self, a, w):
        return a @ w

    def project(self, a, q):
        return q.T @ a

    def omega_rows(self, row0, nrows, total_rows, cols, seed, stream):
        return oracle.gaussian_from_philox(total_rows, cols, seed, stream)[row0:row0 + nrows].astype(np.float64)

    def cholqr(self, y):
        q, r = np.linalg.qr(y)
        return q * np.where(np.diag(r) < 0, -1.0, 1.0)

    def syev(self, w):
        lam, v = np.linalg.eigh(0.5 * (w + w.T))
        return lam[::-1], v[:, ::-1]

    def to_host(self, t):
        return np.asarray(t, dtype=np.float64)

    def from_host(self, a, dtype="float32"):
        return np.asarray(a, dtype=np.float64)

    def allreduce(self, t, group):
        import torch
        import torch.distributed as dist
        tt = torch.from_numpy(np.ascontiguousarray(t, dtype=np.float64))
        dist.all_reduce(tt, group=group)
        return tt.numpy()

    def allgather_cols(self, a, group):
        import torch
        import torch.distributed as dist
        world = dist.get_world_size(group)
        mine = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T))
        blocks = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(blocks, mine, group=group)
        return torch.cat(blocks, dim=0).numpy().T


SHAPE = [12, 12, 10, 8, 16]
RANKS = [1, 10, 10, 8, 6, 1]


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
        cores, used = sharded.tt_svd_sharded(_local_block(x, world, rank), list(x.shape), RANKS, oversample=6,
                                             power_iters=1, seed=77, backend=NumpyBackend())
        np.savez(os.path.join(out_dir, f"w{world}_r{rank}.npz"), *cores, used=np.array(used))
    finally:
        dist.destroy_process_group()


def _run(world, x, out_dir):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), x, out_dir), nprocs=world, join=True)
    res = []
    for r in range(world):
        f = np.load(os.path.join(out_dir, f"w{world}_r{r}.npz"))
        res.append(([f[f"arr_{k}"] for k in range(len(SHAPE))], list(f["used"])))
    return res


@pytest.fixture(scope="module")
def sharded_runs(tmp_path_factory):
    x = oracle.make_tt_tensor(SHAPE, RANKS, 1e-6, seed=41).astype(np.float64)
    d = str(tmp_path_factory.mktemp("sharded"))
    return x, _run(1, x, d), _run(2, x, d)


def test_sharded_ranks_agree_and_match_one_rank(sharded_runs):
    """Both ranks end with the same cores, and two ranks reproduce the one-rank chain: the
    all-reduced Grams and sketches equal the unsharded ones up to summation order, and each
    rank draws exactly its rows of the one Gaussian test matrix."""
    x, one, two = sharded_runs
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
    x, one, two = sharded_runs
    ocores, _ = oracle.tt_svd(x, RANKS, method="gram")
    oerr = oracle.rel_error(x, oracle.tt_full(ocores))
    err = oracle.rel_error(x, oracle.tt_full(two[0][0]))
    assert abs(err - oerr) < 1e-6, (err, oerr)


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
