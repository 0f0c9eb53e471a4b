"""Column-sharded TT-SVD and TR-SVD over several GPUs (one process per GPU, torch.distributed).

Every unfolding of the chain is the column-major matrix (r_{k-1} n_k) x (n_{k+1} ... n_d [r0]),
and its columns run over the last mode i_d slowest (before the ring's bond r0, which the 231
permute moves behind it).  Splitting i_d into P contiguous blocks therefore gives each rank a
fixed set of columns of every unfolding (one contiguous block for a train, r0 strided blocks for
a ring), and the in-place reshape from one unfolding to the next stays local.  Per step the ranks
exchange only small matrices:

* exact step (small side <= 64 rows, or <= 128 when a sketch would cover half of it): all-reduce
  of the m x m Gram A A^T;
* EDrSVD step: all-reduce of the sketch Y = A Omega (m x ks; each rank generates the rows of the
  Gaussian Omega that belong to its columns, so Omega is the one a single GPU would draw), of the
  Gram Z^T Z of the power-iteration basis (ks x ks) and of the Gram B B^T (ks x ks);
* a step whose columns are few (<= 64): all-gather of the unfolding (m x cols, small);
* the last core: all-gather of the remaining r_{d-1} x n_d [r0] data.

The small factorisations (CholeskyQR2, eigen-solves, the inverse square root that
orthonormalises the distributed power basis) run redundantly on every rank, on its GPU, from
identical all-reduced inputs, so every rank ends with the same cores; nothing but the finished
cores is copied to the host.  The reference splits only unfolding 1 over GPUs, through a reduce to
GPU 0 and peer copies (ttdec6_multiGPUs_2.cu:662-776; TR: trdec6_multiGPUs_2.cu:742).

All arithmetic goes through a backend object: ``DeviceBackend`` calls the library's CUDA kernels
on the rank's GPU; the tests substitute a NumPy backend whose arrays refuse host arithmetic, which
checks that the chain itself computes nothing outside the backend.
"""
from __future__ import annotations

import numpy as np


def _small_exact(m: int, cols: int, r_eff: int, s: int) -> bool:
    """Same rule as the single-GPU plan: exact Gram-eigen for small sides <= 64, or <= 128 when
    a sketch would cover half of it anyway."""
    mn = min(m, cols)
    return mn <= 64 or (mn <= 128 and 2 * (r_eff + s) >= mn)


class DeviceBackend:
    """Bulk and small operations on the rank's GPU through libttrsvd (column-major CUDA
    tensors); elementwise steps (column scaling, sign flips, slicing) are torch tensor ops."""

    def __init__(self, device=None, gemm="auto"):
        import torch
        import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
        self.torch = torch
        self.ttr = ttr
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.gemm = gemm

    # layout
    def matrix(self, flat, rows, cols):
        """Column-major (rows x cols) view of a flat device buffer."""
        return flat[: rows * cols].view(cols, rows).t()

    def flat(self, a):
        return a.float().t().contiguous().reshape(-1)

    def cols(self, a, c0, c1):
        """Columns c0..c1-1 (a column-major copy)."""
        return a[:, c0:c1].t().contiguous().t()

    def vcat(self, blocks):
        """Stack (r_i x c) matrices vertically (column-major result)."""
        return self.torch.cat(list(blocks), dim=0).t().contiguous().t()

    def pad_cols(self, a, n):
        rows, c = a.shape
        if c >= n:
            return a
        out = self.torch.zeros((n, rows), dtype=a.dtype, device=a.device).t()
        out[:, :c] = a
        return out

    def permute231(self, flat, r0, r1, n):
        return self.ttr.permute231(flat, r0, r1, n)

    # bulk passes (library kernels)
    def gram_rows(self, a):
        return self.ttr.gram_rows(a, "tc" if self.gemm != "fp32" and a.shape[1] >= (1 << 16) else "fp32")

    def gram_cols(self, a):
        return self.ttr.gram_tall(a)

    def sketch(self, a, w):
        return self.ttr.sketch(a.float(), w.float(), self.gemm)   # A W (FP64)

    def project(self, a, q):
        return self.ttr.project(a, q.float(), self.gemm)          # Q^T A (N x n)

    def omega_rows(self, row0, nrows, total_rows, cols, seed, stream):
        from . import _lib
        import ctypes as C
        out = self.torch.empty((cols, nrows), dtype=self.torch.float32, device=self.device).t()
        _lib.check(self.ttr.lib().tt_k_gaussian_rows(self.ttr._ctx_for(self.device.index),
                                                      C.c_void_p(out.data_ptr()), row0, nrows, total_rows, cols,
                                                      nrows, seed, stream))
        return out

    # small factorisations (library kernels)
    def cholqr(self, y):
        q, _ = self.ttr.cholqr2(y.float())
        return q

    def syev(self, w):
        ev, vec, _ = self.ttr.syev(w)
        return ev, vec

    def inv_sqrt_psd(self, w, rel_floor=1e-12):
        """W^(-1/2) on the range of W (eigen-directions below rel_floor of the largest dropped)."""
        ev, vec = self.syev(w)
        keep = ev > rel_floor * ev[0].clamp(min=1e-300)
        s = self.torch.where(keep, ev.clamp(min=1e-300).rsqrt(), self.torch.zeros_like(ev))
        return self.sketch(vec * s[None, :], vec.t().contiguous().t())

    # elementwise
    def canon(self, u):
        """Columns signed so their largest-magnitude entry is positive (lowest row on ties);
        returns (u, signs)."""
        idx = self.torch.argmax(u.abs(), dim=0)
        v = u.gather(0, idx[None, :])[0]
        sg = self.torch.where(v < 0, -1.0, 1.0).to(u.dtype)
        return u * sg[None, :], sg

    def scale_cols(self, a, s):
        return a * s[None, :].to(a.dtype)

    def scale_rows(self, a, s):
        return a * s[:, None].to(a.dtype)

    def sigma(self, ev, r):
        return ev[:r].clamp(min=0.0).sqrt()

    def recip(self, s):
        return self.torch.where(s > 0, 1.0 / s.clamp(min=1e-300), self.torch.zeros_like(s))

    def head(self, v, r):
        return v[:, :r].t().contiguous().t()

    def t(self, a):
        return a.t()

    # collectives
    def allreduce(self, t, group):
        """In-place sum over the ranks; column-major matrices are reduced through their
        (contiguous) transpose, which shares the storage."""
        import torch.distributed as dist
        if t.is_contiguous():
            dist.all_reduce(t, group=group)
            return t
        if t.dim() == 2 and t.t().is_contiguous():
            dist.all_reduce(t.t(), group=group)
            return t
        c = t.contiguous()
        dist.all_reduce(c, group=group)
        return c

    def allgather_cols(self, a, group):
        """Concatenate the ranks' column blocks (rank order) of a (rows x cols_local) matrix."""
        import torch.distributed as dist
        world = dist.get_world_size(group)
        mine = a.t().contiguous()
        blocks = [self.torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(blocks, mine, group=group)
        return self.torch.cat(blocks, dim=0).t()

    def to_host(self, t):
        return t.double().cpu().numpy()


def _rank_info(group):
    import torch.distributed as dist
    if dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def _chain(x_local, shape, ranks, ring, oversample, power_iters, seed, group, be):
    """The sharded sequential chain (TT when not ring).  Returns backend bases per step, the
    last data block and bookkeeping."""
    world, rank = _rank_info(group)
    d = len(shape)
    if shape[-1] % world:
        raise ValueError(f"last mode {shape[-1]} does not split over {world} ranks")
    nloc = shape[-1] // world
    r0 = ranks[0] if ring else 1
    s = max(0, int(oversample))
    data = x_local
    size_loc = int(np.prod(shape[:-1])) * nloc
    r_prev = 1
    bases, used = [], [ranks[0] if ring else 1]
    for k in range(d - 1):
        first_ring = ring and k == 0
        m = r_prev * shape[k]
        cols_loc = size_loc // m
        cols = cols_loc * world
        a = be.matrix(data, m, cols_loc)
        rq = ranks[0] * ranks[1] if first_ring else ranks[k + 1]
        r_eff = min(rq, m, cols)
        # columns of this unfolding per bond index a0 of the ring: (modes k+2 .. d-1) x i_d
        mid = int(np.prod(shape[k + 1:d - 1])) if k + 1 < d - 1 else 1
        rs0 = 1 if first_ring else r0  # r0 blocks of columns after the 231 permute
        if _small_exact(m, cols, r_eff, s) and m <= cols:
            w = be.allreduce(be.gram_rows(a), group)
            _, vec = be.syev(w)
            u, _ = be.canon(be.head(vec, r_eff))
            nxt = be.project(a, u)                                    # r_eff x cols_loc
        elif _small_exact(m, cols, r_eff, s):
            full = be.allgather_cols(a, group)                        # m x cols (rank-major)
            ev, v = be.syev(be.gram_cols(full))                       # A^T A (cols x cols)
            sig = be.sigma(ev, r_eff)
            vr = be.head(v, r_eff)
            u, sg = be.canon(be.sketch(full, be.scale_cols(vr, be.recip(sig))))  # A V / sigma
            nxt_full = be.scale_rows(be.scale_rows(be.t(vr), sig), sg)  # r_eff x cols (rank-major)
            nxt = be.cols(nxt_full, rank * cols_loc, (rank + 1) * cols_loc)
        else:
            ks = min(r_eff + s, m, cols, 128)
            # this rank's rows of the one Gaussian Omega: per ring bond a0, a contiguous range
            blocks = [be.omega_rows(mid * (rank * nloc + shape[-1] * a0), mid * nloc, cols, ks, seed, k)
                      for a0 in range(rs0)]
            om = blocks[0] if rs0 == 1 else be.vcat(blocks)
            y = be.allreduce(be.sketch(a, om), group)
            q = be.cholqr(y)
            for _ in range(power_iters):
                zt = be.project(a, q)                                 # Z^T = Q^T A (ks x cols_loc)
                wz = be.allreduce(be.gram_rows(zt), group)            # Z^T Z (ks x ks)
                z = be.sketch(be.t(zt), be.inv_sqrt_psd(wz))          # Z (Z^T Z)^(-1/2), orthonormal
                y = be.allreduce(be.sketch(a, z), group)
                q = be.cholqr(y)
            b = be.project(a, q)                                      # B = Q^T A (ks x cols_loc)
            _, vec = be.syev(be.allreduce(be.gram_rows(b), group))   # B B^T
            e = be.head(vec, r_eff)
            u, sg = be.canon(be.sketch(q, e))                         # U = Q E_r
            nxt = be.project(b, be.scale_cols(e, sg))                 # E_r^T B (r_eff x cols_loc)
        if first_ring:
            u = be.pad_cols(u, rq)                                    # bond split q = a + r0 b
            nxt_full_rows = be.pad_cols(be.t(nxt), rq)                # rows beyond r_eff are zero
            flat = be.flat(be.t(nxt_full_rows))                       # (r0, r1, cols_loc)
            data = be.permute231(flat, ranks[0], ranks[1], cols_loc)  # (r1, cols_loc, r0)
            r_prev = ranks[1]
            size_loc = rq * cols_loc
            used.append(ranks[1])
        else:
            data = be.flat(nxt)
            size_loc = r_eff * cols_loc
            r_prev = r_eff
            used.append(r_eff)
        bases.append(u)
    last = be.matrix(data, r_prev, size_loc // r_prev)
    return bases, last, used, world, rank, nloc, r0


def tt_svd_sharded(x_local, shape, ranks, *, oversample=8, power_iters=0, seed=1234, group=None,
                   backend=None):
    """TT-SVD of a tensor whose last mode is split evenly over the ranks of ``group``.

    ``x_local``: this rank's block, the column-major flat tensor of shape
    (n_1, ..., n_{d-1}, n_d / P) holding i_d in [rank n_d / P, (rank + 1) n_d / P).  Returns the
    cores (host NumPy arrays, logical shape (r_{k-1}, n_k, r_k), identical on every rank) and the
    ranks used (requested ranks above what an unfolding carries are reduced).
    """
    be = backend or DeviceBackend()
    bases, last, used, world, rank, nloc, _ = _chain(x_local, shape, ranks, False, oversample, power_iters,
                                                      seed, group, be)
    cores = []
    for k, u in enumerate(bases):
        cores.append(be.to_host(u).reshape(used[k], shape[k], used[k + 1], order="F"))
    lastf = be.to_host(be.allgather_cols(last, group))               # r x n_d
    cores.append(lastf.reshape(used[-1], shape[-1], 1, order="F"))
    used.append(1)
    return cores, used


def tr_svd_sharded(x_local, shape, ranks, *, oversample=8, power_iters=0, seed=1234, group=None,
                   backend=None):
    """TR-SVD (bond ranks [r0, r1, ..., r_{d-1}, r0]) of a tensor whose last mode is split evenly
    over the ranks of ``group``, as :func:`tt_svd_sharded`.  Step 1 factorises unfolding 1 at
    rank r0 r1 (zero-padded beyond what it carries) and moves r0 behind i_d (the 231 permute,
    TR6:49-58), which keeps every later unfolding's columns on the rank that owns their i_d.
    Returns the cores (host, logical shape (r_{k-1}, n_k, r_k) with r_d = r0) and the ranks."""
    be = backend or DeviceBackend()
    bases, last, used, world, rank, nloc, r0 = _chain(x_local, shape, ranks, True, oversample, power_iters,
                                                       seed, group, be)
    n1, r1 = shape[0], ranks[1]
    g1 = be.to_host(bases[0]).reshape(n1, r0, r1, order="F").transpose(1, 0, 2)   # (r0, n1, r1)
    cores = [np.ascontiguousarray(g1)]
    for k in range(1, len(bases)):
        cores.append(be.to_host(bases[k]).reshape(used[k], shape[k], used[k + 1], order="F"))
    # last data: rank blocks of (r_{d-1}) x (nloc x r0) columns -> (r_{d-1}, n_d, r0)
    g = be.to_host(be.allgather_cols(last, group))  # r x (i_dl, a0, rank), i_dl fastest
    rl = used[-1]
    g = g.reshape(rl, nloc, r0, world, order="F").transpose(0, 1, 3, 2).reshape(rl, world * nloc, r0, order="F")
    cores.append(g)
    used.append(r0)
    return cores, used
