"""Column-sharded TT-SVD over several GPUs (one process per GPU, torch.distributed).

Every unfolding of the TT chain is the column-major matrix (r_{k-1} n_k) x (n_{k+1} ... n_d), and
its columns run over the last mode i_d slowest.  Splitting i_d into P contiguous blocks therefore
gives each rank a contiguous column block of every unfolding, and the in-place reshape from one
unfolding to the next stays local.  Per step the ranks exchange only small matrices:

* exact step (small side <= 64 rows): all-reduce of the m x m Gram A A^T;
* EDrSVD step: all-reduce of the sketch Y = A Omega (m x ks; each rank generates the rows of the
  Gaussian Omega that belong to its columns, so Omega is the one a single GPU would draw), of the
  Gram of the power-iteration basis Z (ks x ks), and of the Gram B B^T (ks x ks);
* a step whose columns are few (<= 64): all-gather of the unfolding (m x cols, small);
* the last core: all-gather of the remaining r_{d-1} x n_d data.

The small factorisations (CholeskyQR2, Jacobi) run redundantly on every rank from identical
all-reduced inputs, so every rank ends with the same cores.  The reference splits only unfolding 1
over GPUs, through a reduce to GPU 0 and peer copies (ttdec6_multiGPUs_2.cu:662-776).

The bulk work goes through a backend: ``DeviceBackend`` calls the library's CUDA kernels on the
rank's GPU; tests substitute a NumPy backend to check the orchestration with gloo on the CPU.
"""
from __future__ import annotations

import numpy as np


def _small_exact(m: int, cols: int, r_eff: int, s: int) -> bool:
    """Same rule as the single-GPU plan: exact Gram-eigen for small sides <= 64, or <= 128 when
    a sketch would cover half of it anyway."""
    mn = min(m, cols)
    return mn <= 64 or (mn <= 128 and 2 * (r_eff + s) >= mn)


def _canon(u: np.ndarray):
    """Signs making each column's largest-magnitude entry positive (lowest row on ties)."""
    idx = np.argmax(np.abs(u), axis=0)
    return np.where(u[idx, np.arange(u.shape[1])] < 0, -1.0, 1.0)


class DeviceBackend:
    """Bulk operations on the rank's GPU through libttrsvd (column-major CUDA tensors)."""

    def __init__(self, device=None, gemm="auto"):
        import torch
        import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
        self.torch = torch
        self.ttr = ttr
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.gemm = gemm

    def matrix(self, flat, rows, cols):
        """Column-major (rows x cols) view of a flat device buffer."""
        return flat[: rows * cols].view(cols, rows).t()

    def flat(self, a):
        return a.t().contiguous().reshape(-1)

    def transpose(self, a):
        return a.t()

    def gram_rows(self, a):
        return self.ttr.gram_rows(a, "tc" if self.gemm != "fp32" and a.shape[1] >= (1 << 16) else "fp32")

    def sketch(self, a, w):
        return self.ttr.sketch(a, w, self.gemm)

    def project(self, a, q):
        return self.ttr.project(a, q, self.gemm)  # (N x n), Q^T A

    def omega_rows(self, row0, nrows, total_rows, cols, seed, stream):
        from . import _lib
        import ctypes as C
        out = self.torch.empty((cols, nrows), dtype=self.torch.float32, device=self.device).t()
        _lib.check(self.ttr.lib().tt_k_gaussian_rows(self.ttr._ctx_for(self.device.index),
                                                      C.c_void_p(out.data_ptr()), row0, nrows, total_rows, cols,
                                                      nrows, seed, stream))
        return out

    def cholqr(self, y):
        q, _ = self.ttr.cholqr2(y.float())
        return q

    def syev(self, w):
        ev, vec, _ = self.ttr.syev(w)
        return ev, vec

    def to_host(self, t):
        return t.double().cpu().numpy()

    def from_host(self, a, dtype="float32"):
        t = self.torch.from_numpy(np.asfortranarray(a)).to(self.device)
        t = t.float() if dtype == "float32" else t.double()
        return t.t().contiguous().t()  # column-major

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
        blocks = [self.torch.empty_like(a.t().contiguous()) for _ in range(world)]
        dist.all_gather(blocks, a.t().contiguous(), group=group)
        return self.torch.cat(blocks, dim=0).t()


def tt_svd_sharded(x_local, shape, ranks, *, oversample=8, power_iters=0, seed=1234, group=None,
                   backend=None):
    """TT-SVD of a tensor whose last mode is split evenly over the ranks of ``group``.

    ``x_local``: this rank's block, the column-major flat tensor of shape
    (n_1, ..., n_{d-1}, n_d / P) holding i_d in [rank n_d / P, (rank + 1) n_d / P).  Returns the
    cores (host NumPy arrays, logical shape (r_{k-1}, n_k, r_k), identical on every rank) and the
    ranks used (requested ranks above what an unfolding carries are reduced).
    """
    import torch.distributed as dist
    be = backend or DeviceBackend()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    d = len(shape)
    if shape[-1] % world:
        raise ValueError(f"last mode {shape[-1]} does not split over {world} ranks")
    nloc = shape[-1] // world
    s = max(0, int(oversample))
    size_loc = int(np.prod(shape[:-1])) * nloc
    data = x_local
    r_prev = 1
    cores, used = [], [1]
    for k in range(d - 1):
        m = r_prev * shape[k]
        cols_loc = size_loc // m
        cols = cols_loc * world
        a = be.matrix(data, m, cols_loc)
        r_eff = min(ranks[k + 1], m, cols)
        if _small_exact(m, cols, r_eff, s) and m <= cols:
            w = be.allreduce(be.gram_rows(a), group)
            ev, vec = be.syev(w)
            u = be.to_host(vec)[:, :r_eff]
            u = u * _canon(u)
            nxt = be.project(a, be.from_host(u))  # r x cols_loc
        elif _small_exact(m, cols, r_eff, s):
            full = be.allgather_cols(a, group)  # m x cols
            fh = be.to_host(full)
            w = fh.T @ fh
            lam, v = np.linalg.eigh(w)
            lam, v = lam[::-1][:r_eff], v[:, ::-1][:, :r_eff]
            sig = np.sqrt(np.maximum(lam, 0.0))
            u = fh @ v / np.where(sig > 0, sig, 1.0)
            sg = _canon(u)
            u = u * sg
            nxt_full = (sg * sig)[:, None] * v.T  # r x cols
            nxt = be.from_host(np.ascontiguousarray(nxt_full[:, rank * cols_loc:(rank + 1) * cols_loc]))
        else:
            ks = min(r_eff + s, m, cols, 128)
            om = be.omega_rows(rank * cols_loc, cols_loc, cols, ks, seed, k)
            y = be.allreduce(be.sketch(a, om), group)
            q = be.cholqr(y)
            for _ in range(power_iters):
                zt = be.project(a, q)                         # Z^T = Q^T A (ks x cols_loc)
                wz = be.allreduce(be.gram_rows(zt), group)     # Z^T Z (ks x ks)
                # Z^T Z is singular to working precision when A's rank is below ks; a shift of
                # 1e-12 of its trace keeps the Cholesky factor finite (R^-1 only conditions Z)
                wzh = be.to_host(wz)
                wzh = 0.5 * (wzh + wzh.T)
                shift = 1e-12 * max(float(np.trace(wzh)), 1e-300)
                rz = np.linalg.cholesky(wzh + shift * np.eye(ks)).T  # upper
                z = be.sketch(be.transpose(zt), be.from_host(np.linalg.inv(rz)))  # Z R^-1
                y = be.allreduce(be.sketch(a, z), group)
                q = be.cholqr(y)
            b = be.project(a, q)                              # ks x cols_loc
            w = be.allreduce(be.gram_rows(b), group)          # B B^T
            ev, vec = be.syev(w)
            e = be.to_host(vec)[:, :r_eff]
            u = be.to_host(q) @ e
            sg = _canon(u)
            u, e = u * sg, e * sg
            nxt = be.project(b, be.from_host(e))              # r x cols_loc
        cores.append(np.asarray(u, dtype=np.float64).reshape(r_prev, shape[k], r_eff, order="F"))
        used.append(r_eff)
        data = be.flat(nxt)
        size_loc = r_eff * cols_loc
        r_prev = r_eff
    last = be.to_host(be.allgather_cols(be.matrix(data, r_prev, nloc), group))  # r x n_d
    cores.append(last.reshape(r_prev, shape[-1], 1, order="F"))
    used.append(1)
    return cores, used
