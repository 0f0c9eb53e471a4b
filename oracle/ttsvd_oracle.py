"""NumPy restatement of the reference's TT-SVD / TR-SVD algorithms (FP64 by default).

TEST INFRASTRUCTURE ONLY: the FP64 results the CUDA path is compared with, and
the timed CPU baseline.  The product never imports this file.

Parity status: PINNED.  ``tr_svd(..., convention="python")`` and
``tt_svd(..., convention="python")`` are checked bit-for-bit-equivalent
(same LAPACK SVD, same reshapes) against the reference's own Python TR-SVD
``trdecomposition/high_order_GPUs/python_GPUs/T3F.py:38-79`` executed in this
container through a NumPy stand-in for the four TensorFlow calls it makes;
the golden vectors live in ``tests/golden/`` together with the script that
produced them.  The ``convention="gpu"`` variants differ only in index order
(column-major unfoldings, ``q = a + r0*b`` bond split, the ``231`` permute of
``TR6:49-58``) and are checked against the python convention through
order-independent properties (singular values, reconstruction error).

Conventions (reference GPU code, ``TT6:817-927``, ``TR6:827-1004``):
  * tensors are column-major, mode 1 fastest: X(i1..id) at i1 + n1*(i2 + n2*(...));
  * unfolding j of the TT chain is the (r_{j-1} n_j) x (n_{j+1}...n_d) column-major matrix;
  * after step j the projected factor S V^T (r_j x rest) is re-read in place as the
    next unfolding, so the TT reshape costs nothing;
  * core k is stored as a column-major (r_{k-1}, n_k, r_k) array.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "unfold", "canon_signs", "truncated_svd", "gram_eig", "tt_svd", "tr_svd", "tt_full", "tr_full",
    "rel_error", "tt_random_cores", "tr_random_cores", "add_noise", "make_tt_tensor",
    "make_tr_tensor", "edrsvd_plain", "edrsvd_gram", "gram_eig_step", "ttdec6_gram",
    "trdec6_gram", "philox4x32_10", "gaussian_from_philox", "ref_uniform_tt_tensor",
    "tt_flops_model", "tt_svd_eps",
]


# ----------------------------------------------------------------------------
# basic linear algebra
# ----------------------------------------------------------------------------
def unfold(flat: np.ndarray, m: int, n: int) -> np.ndarray:
    """Column-major (m x n) view of a flat buffer (``TT6:817-818``)."""
    return flat.reshape(m, n, order="F")


def canon_signs(u: np.ndarray, svt: np.ndarray, k: int):
    """Sign convention of the CUDA chain: for each of the first k columns of the basis u, the
    entry of largest magnitude (lowest row on ties) is made positive; the matching row of
    svt is negated with it.  TR-SVD's later unfoldings depend on these signs."""
    for a in range(min(k, u.shape[1])):
        col = u[:, a]
        i = int(np.argmax(np.abs(col)))
        if col[i] < 0:
            u[:, a] = -col
            svt[a] = -svt[a]
    return u, svt


def truncated_svd(a: np.ndarray, r: int):
    """Thin SVD truncated to ``r`` (``T3F.py:41-45``: svd -> u[:, :r], s[:r], v[:, :r])."""
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    r = min(r, s.size)
    return u[:, :r], s, vt[:r]


def gram_eig(a: np.ndarray, r: int):
    """Top-``r`` left singular subspace from the Gram matrix A A^T.

    Restates ``longMatrixSVD_Eign_once_device`` (``TT6:510-536``): Gram ``A A^T``
    (``TT6:388-401``), symmetric eigensolver (``basicEig`` ``TT6:334-385``), the
    eigenvectors taken in descending order (``matrixInvertColumn`` ``TT6:274-290``)
    and the projection ``G^T A`` (``TT6:424-442``).  Returns (G, sigma, G^T A).
    Requested ranks beyond the row count are zero-padded instead of read out of
    bounds (the reference's ``matrixInvertColumn_kernel`` reads past the matrix there).
    """
    w = a @ a.T
    lam, v = np.linalg.eigh(w)
    lam = lam[::-1]
    v = v[:, ::-1]
    m = a.shape[0]
    g = np.zeros((m, r), dtype=a.dtype)
    k = min(r, m)
    g[:, :k] = v[:, :k]
    return g, np.sqrt(np.maximum(lam, 0.0)), g.T @ a


# ----------------------------------------------------------------------------
# TT-SVD / TR-SVD drivers
# ----------------------------------------------------------------------------
def tt_svd(x: np.ndarray, ranks, method: str = "svd", convention: str = "gpu", dtype=np.float64):
    """Sequential TT-SVD with fixed target ranks.

    ``convention="gpu"``: column-major chain of ``ttdec_half_lu_device_6`` (``TT6:799-958``).
    ``convention="python"``: row-major chain of the repo's Python TR-SVD with r0 = r_d = 1
    (``T3F.py:38-79``), i.e. the C-order reshapes of that file.
    Returns (cores, sigmas): cores[k] has shape (r_{k-1}, n_k, r_k) (logical index order
    a, i, b for both conventions); sigmas[k] are all singular values of unfolding k+1.
    """
    ranks = list(ranks)
    n = list(x.shape)
    d = len(n)
    assert len(ranks) == d + 1 and ranks[0] == 1 and ranks[-1] == 1
    order = "F" if convention == "gpu" else "C"
    flat = np.asarray(x, dtype=dtype).ravel(order=order)
    cores, sigmas = [], []
    r_prev = 1
    for k in range(d - 1):
        m = r_prev * n[k]
        cols = flat.size // m
        a = flat.reshape(m, cols, order=order)
        if method == "svd":
            u, s, vt = truncated_svd(a, ranks[k + 1])
            r = u.shape[1]
            svt = s[:r, None] * vt
        else:
            u, s, svt = gram_eig(a, ranks[k + 1])
            r = u.shape[1]
        sigmas.append(s)
        if convention == "gpu":
            u, svt = canon_signs(u.copy(), svt.copy(), min(r, a.shape[0], a.shape[1]))
            cores.append(u.reshape(r_prev, n[k], r, order="F"))
        else:
            cores.append(u.reshape(r_prev, n[k], r, order="C"))
        flat = svt.ravel(order=order)
        r_prev = r
    if convention == "gpu":
        cores.append(flat.reshape(r_prev, n[-1], 1, order="F"))
    else:
        cores.append(flat.reshape(r_prev, n[-1], 1, order="C"))
    return cores, sigmas


def tr_svd(x: np.ndarray, ranks, method: str = "svd", convention: str = "gpu", dtype=np.float64):
    """Sequential TR-SVD (tensor ring) with fixed bond ranks ``ranks = [r0, r1, ..., r_{d-1}, r0]``.

    Step 1 factorises unfolding 1 at rank r0*r1 and moves the r0 bond to the slowest
    position.  ``convention="gpu"`` follows ``TR6:827-1004``: bond index q = a + r0*b and the
    ``tensorToMode231`` permute (r0, r1, N) -> (r1, N, r0) of ``TR6:49-58``.
    ``convention="python"`` follows ``T3F.py:38-79``: q = a*r1 + b and transpose (1, 2, 0)
    on C-order reshapes.  Ranks above what unfolding 1 can carry are zero-padded.
    Returns (cores, sigmas); cores[k] has logical shape (r_{k-1}, n_k, r_k) with r_d = r0.
    """
    ranks = list(ranks)
    n = list(x.shape)
    d = len(n)
    assert len(ranks) == d + 1 and ranks[0] == ranks[-1]
    r0, r1 = ranks[0], ranks[1]
    order = "F" if convention == "gpu" else "C"
    flat = np.asarray(x, dtype=dtype).ravel(order=order)
    ncols = flat.size // n[0]
    a = flat.reshape(n[0], ncols, order=order)
    q = r0 * r1
    if method == "svd":
        u, s, vt = np.linalg.svd(a, full_matrices=False)
        k = min(q, s.size)
        uq = np.zeros((n[0], q), dtype=a.dtype)
        uq[:, :k] = u[:, :k]
        svt = np.zeros((q, ncols), dtype=a.dtype)
        svt[:k] = s[:k, None] * vt[:k]
    else:
        uq, s, svt = gram_eig(a, q)
    sigmas = [s]
    if convention == "gpu":
        uq, svt = canon_signs(uq.copy(), svt.copy(), min(q, n[0], ncols))
        g1 = uq.reshape(n[0], r0, r1, order="F").transpose(1, 0, 2)  # (r0, n1, r1)
        t = svt.reshape(r0, r1, ncols, order="F").transpose(1, 2, 0)  # (r1, N, r0)
        flat = t.ravel(order="F")
    else:
        g1 = uq.reshape(n[0], r0, r1, order="C").transpose(1, 0, 2)
        t = svt.reshape(r0, r1, ncols, order="C").transpose(1, 2, 0)
        flat = t.ravel(order="C")
    cores = [g1]
    r_prev = r1
    for k in range(1, d - 1):
        m = r_prev * n[k]
        cols = flat.size // m
        a = flat.reshape(m, cols, order=order)
        if method == "svd":
            u, s, vt = truncated_svd(a, ranks[k + 1])
            r = u.shape[1]
            svt = s[:r, None] * vt
        else:
            u, s, svt = gram_eig(a, ranks[k + 1])
            r = u.shape[1]
        sigmas.append(s)
        if convention == "gpu":
            u, svt = canon_signs(u.copy(), svt.copy(), min(r, a.shape[0], a.shape[1]))
        cores.append(u.reshape(r_prev, n[k], r, order=order))
        flat = svt.ravel(order=order)
        r_prev = r
    cores.append(flat.reshape(r_prev, n[-1], r0, order=order))
    return cores, sigmas


def _merge_right(cores, order: str):
    """Contract cores[1:] into one (r1, n2*...*nd, r_d) array (mode 2 fastest for 'F')."""
    m = cores[1]
    for g in cores[2:]:
        ra, na, rb = m.shape
        _, nb, rc = g.shape
        t = np.tensordot(m, g, axes=([2], [0]))  # (ra, na, nb, rc)
        m = t.reshape(ra, na * nb, rc, order=order)
    return m


def tt_full(cores, convention: str = "gpu") -> np.ndarray:
    """Reconstruct X from TT cores (restates ``calMSE``'s right-to-left contraction ``TT6:134-182``)."""
    return tr_full(cores, convention)


def tt_svd_eps(x: np.ndarray, eps: float, max_ranks=None, dtype=np.float64):
    """TT-SVD with delta-truncation (Oseledets, TT-SVD algorithm): every unfolding keeps the
    smallest rank r whose discarded squared singular values sum to at most
    eps^2 ||X||_F^2 / (d - 1), capped by ``max_ranks``; then ||X - X^|| <= eps ||X||.
    Column-major chain with canonical signs (the GPU convention).  Returns (cores, ranks)."""
    n = list(x.shape)
    d = len(n)
    flat = np.asarray(x, dtype=dtype).ravel(order="F")
    delta2 = eps * eps * float(np.sum(flat * flat)) / (d - 1)
    cores, ranks = [], [1]
    r_prev = 1
    for k in range(d - 1):
        m = r_prev * n[k]
        a = flat.reshape(m, flat.size // m, order="F")
        u, s, vt = np.linalg.svd(a, full_matrices=False)
        cap = s.size if max_ranks is None else min(s.size, max_ranks[k + 1])
        tail = np.concatenate([np.cumsum((s ** 2)[::-1])[::-1], [0.0]])  # tail[r] = sum_{i>=r} s_i^2
        r = 1
        while r < cap and tail[r] > delta2:
            r += 1
        u, svt = canon_signs(u[:, :r].copy(), (s[:r, None] * vt[:r]).copy(), r)
        cores.append(u.reshape(r_prev, n[k], r, order="F"))
        flat = svt.ravel(order="F")
        r_prev = r
        ranks.append(r)
    cores.append(flat.reshape(r_prev, n[-1], 1, order="F"))
    ranks.append(1)
    return cores, ranks


def tr_full(cores, convention: str = "gpu") -> np.ndarray:
    """Reconstruct X from ring cores: X = Tr(G1(i1) ... Gd(id)) (``T3F.py:27-36``, ``TR6:175-229``)."""
    order = "F" if convention == "gpu" else "C"
    shape = [g.shape[1] for g in cores]
    if len(cores) == 1:
        g = cores[0]
        return np.einsum("aia->i", g).reshape(shape)
    m = _merge_right(cores, order)  # (r1, N, r0)
    g1 = cores[0]  # (r0, n1, r1)
    x = np.einsum("aib,bja->ij", g1, m)  # (n1, N)
    return x.reshape(shape, order=order)


def rel_error(x: np.ndarray, xh: np.ndarray) -> float:
    """||X - X_hat||_F / ||X||_F in FP64 (the quantity ``calMSE`` prints as "MSE", ``TT6:178-181``)."""
    x = np.asarray(x, dtype=np.float64)
    xh = np.asarray(xh, dtype=np.float64)
    return float(np.linalg.norm((x - xh).ravel()) / np.linalg.norm(x.ravel()))


# ----------------------------------------------------------------------------
# synthetic inputs of the benchmark configurations
# ----------------------------------------------------------------------------
def tt_random_cores(n, ranks, rng, dtype=np.float64):
    """TT cores with i.i.d. N(0,1) entries, core k of shape (r_{k-1}, n_k, r_k)."""
    return [rng.standard_normal((ranks[k], n[k], ranks[k + 1])).astype(dtype) for k in range(len(n))]


def tr_random_cores(n, bond, rng, dtype=np.float64):
    """Ring cores with all bond ranks ``bond`` and i.i.d. N(0,1) entries."""
    d = len(n)
    return [rng.standard_normal((bond, n[k], bond)).astype(dtype) for k in range(d)]


def add_noise(x: np.ndarray, rel: float, rng) -> np.ndarray:
    """X + rel * ||X||_F / sqrt(numel) * N(0,1): Gaussian noise of relative Frobenius size ~rel."""
    if rel == 0:
        return x
    scale = rel * np.linalg.norm(x.ravel()) / np.sqrt(x.size)
    return x + scale * rng.standard_normal(x.shape)


def make_tt_tensor(n, ranks, noise: float, seed: int, dtype=np.float32):
    rng = np.random.default_rng(seed)
    cores = tt_random_cores(n, ranks, rng)
    x = add_noise(tt_full(cores), noise, rng)
    return np.asfortranarray(x.astype(dtype))


def make_tr_tensor(n, bond: int, noise: float, seed: int, dtype=np.float32):
    rng = np.random.default_rng(seed)
    cores = tr_random_cores(n, bond, rng)
    x = add_noise(tr_full(cores), noise, rng)
    return np.asfortranarray(x.astype(dtype))


def ref_uniform_tt_tensor(n, ranks, draw):
    """Order-d analogue of ``generalTTTensor`` (``TT6:185-271``): cores uniform[-1,1) drawn in the
    reference's order (G_{d-1}, G_d first, then G_{d-2}, ..., G_1) from the callable ``draw(size)``,
    contracted right to left.  ``draw`` stands in for the C library ``rand()`` stream."""
    d = len(n)
    sizes = [ranks[k] * n[k] * ranks[k + 1] for k in range(d)]
    cores = [None] * d
    cores[d - 2] = draw(sizes[d - 2]).reshape(ranks[d - 2], n[d - 2], ranks[d - 1], order="F")
    cores[d - 1] = draw(sizes[d - 1]).reshape(ranks[d - 1], n[d - 1], ranks[d], order="F")
    for k in range(d - 3, -1, -1):
        cores[k] = draw(sizes[k]).reshape(ranks[k], n[k], ranks[k + 1], order="F")
    return cores, tt_full(cores)


# ----------------------------------------------------------------------------
# EDrSVD restatements (given the Gaussian test matrix Omega)
# ----------------------------------------------------------------------------
def _qr_q(y: np.ndarray) -> np.ndarray:
    """Explicit Q of a thin Householder QR (``basicQR``: geqrf + orgqr, ``EDR:31-88``)."""
    q, _ = np.linalg.qr(y, mode="reduced")
    return q


def edrsvd_plain(a: np.ndarray, k: int, s: int, p: int, omega: np.ndarray):
    """Plain EDrSVD, ``basicRandSVD`` ``EDR:175-326``.

    Y = A Omega -> Q = qr(Y) -> p x {Z = A^T Q, Q_z = qr(Z), Y = A Q_z, Q = qr(Y)} ->
    B = Q^T A -> SVD(B) = Ut S V^T (``basicSvd`` ``EDR:90-173``) -> U = Q Ut.
    Returns U (m x ks), S (ks), V^T (ks x n).
    """
    ks = k + s
    assert omega.shape == (a.shape[1], ks)
    q = _qr_q(a @ omega)
    for _ in range(p):
        z = _qr_q(a.T @ q)
        q = _qr_q(a @ z)
    b = q.T @ a
    ut, sv, vt = np.linalg.svd(b, full_matrices=False)
    return q @ ut, sv, vt


def edrsvd_gram(a: np.ndarray, k: int, s: int, p: int, omega: np.ndarray):
    """EDrSVD with the Gram-eigen small SVD, ``basicRandSVD_LU`` ``TT3O:557-775``.

    As :func:`edrsvd_plain` up to B = Q^T A, then B B^T (``TT3O:717``) -> eigenvectors in
    descending order (``TT3O:720-728``) -> S V^T = Ut^T B (``TT3O:734``) and U = Q Ut
    (``TT3O:745``).  Returns U (m x ks), sigma (ks), S V^T (ks x n).
    """
    ks = k + s
    assert omega.shape == (a.shape[1], ks)
    q = _qr_q(a @ omega)
    for _ in range(p):
        z = _qr_q(a.T @ q)
        q = _qr_q(a @ z)
    b = q.T @ a
    lam, v = np.linalg.eigh(b @ b.T)
    lam, v = lam[::-1], v[:, ::-1]
    return q @ v, np.sqrt(np.maximum(lam, 0.0)), v.T @ b


def gram_eig_step(a: np.ndarray, r: int):
    """One order-6 step, ``longMatrixSVD_Eign_once_device`` ``TT6:510-536``: returns (G, sigma, G^T A)."""
    return gram_eig(a, r)


def ttdec6_gram(x: np.ndarray, ranks, dtype=np.float64):
    """Order-d TT driver of ``ttdec_half_lu_device_6`` (``TT6:799-958``) with the Gram-eig step."""
    return tt_svd(x, ranks, method="gram", convention="gpu", dtype=dtype)


def trdec6_gram(x: np.ndarray, ranks, dtype=np.float64):
    """Order-d TR driver of ``TR6:827-1004`` with the Gram-eig step and the 231 permute."""
    return tr_svd(x, ranks, method="gram", convention="gpu", dtype=dtype)


# ----------------------------------------------------------------------------
# counter-based Gaussian test matrix (restatement of the device generator)
# ----------------------------------------------------------------------------
_PHILOX_M0 = np.uint64(0xD2511F53)
_PHILOX_M1 = np.uint64(0xCD9E8D57)
_PHILOX_W0 = np.uint32(0x9E3779B9)
_PHILOX_W1 = np.uint32(0xBB67AE85)


def philox4x32_10(counter: np.ndarray, key: tuple[int, int]) -> np.ndarray:
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) on a (N, 4) uint32 counter array.

    Published algorithm: ten rounds of two 32x32->64 multiplies with the constants
    0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule 0x9E3779B9 / 0xBB67AE85.
    """
    c = counter.astype(np.uint32).copy()
    k0 = np.uint32(key[0])
    k1 = np.uint32(key[1])
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = c[:, 0].astype(np.uint64) * _PHILOX_M0
        p1 = c[:, 2].astype(np.uint64) * _PHILOX_M1
        hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
        lo0 = (p0 & mask).astype(np.uint32)
        hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
        lo1 = (p1 & mask).astype(np.uint32)
        n0 = hi1 ^ c[:, 1] ^ k0
        n1 = lo1
        n2 = hi0 ^ c[:, 3] ^ k1
        n3 = lo0
        c = np.stack([n0, n1, n2, n3], axis=1)
        k0 = np.uint32((int(k0) + int(_PHILOX_W0)) & 0xFFFFFFFF)
        k1 = np.uint32((int(k1) + int(_PHILOX_W1)) & 0xFFFFFFFF)
    return c


def gaussian_from_philox(nrows: int, ncols: int, seed: int, stream: int = 0) -> np.ndarray:
    """Column-major (nrows x ncols) N(0,1) matrix of the device generator ``tt_k_gaussian``.

    Flat column-major element e is lane e % 4 of Philox call c = e // 4, whose counter is
    (c mod 2^32, stream, c >> 32, 0) and key (seed mod 2^32, seed >> 32).  The four words
    w0..w3 become u = (w + 0.5) * 2^-32 and two Box-Muller pairs:
    g0, g1 = sqrt(-2 ln u0) (cos, sin)(2 pi u1);  g2, g3 = sqrt(-2 ln u2) (cos, sin)(2 pi u3).
    """
    total = nrows * ncols
    calls = (total + 3) // 4
    ctr = np.zeros((calls, 4), dtype=np.uint32)
    ctr[:, 0] = np.arange(calls, dtype=np.uint64).astype(np.uint32)
    ctr[:, 1] = np.uint32(stream)
    ctr[:, 2] = (np.arange(calls, dtype=np.uint64) >> np.uint64(32)).astype(np.uint32)
    w = philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)).astype(np.float64)
    u = (w + 0.5) * (2.0 ** -32)
    r0 = np.sqrt(-2.0 * np.log(u[:, 0]))
    r1 = np.sqrt(-2.0 * np.log(u[:, 2]))
    g = np.empty((calls, 4))
    g[:, 0] = r0 * np.cos(2 * np.pi * u[:, 1])
    g[:, 1] = r0 * np.sin(2 * np.pi * u[:, 1])
    g[:, 2] = r1 * np.cos(2 * np.pi * u[:, 3])
    g[:, 3] = r1 * np.sin(2 * np.pi * u[:, 3])
    return g.ravel()[:total].reshape(nrows, ncols, order="F")


# ----------------------------------------------------------------------------
# algorithmic work model (the roofline basis)
# ----------------------------------------------------------------------------
def tt_flops_model(n, ranks, ks_extra: int = 8, p: int = 0):
    """Algorithmic FLOPs of one fixed-rank randomized TT-SVD chain (GEMM passes only).

    Per unfolding m x n with target r: exact Gram path when min(m, n) <= r + ks_extra
    (2 m^2 n for the Gram + 2 m r n for the projection); otherwise 2 m n ks (2 + 2p).
    """
    d = len(n)
    total = 0.0
    r_prev = 1
    size = int(np.prod(n))
    for k in range(d - 1):
        m = r_prev * n[k]
        cols = size // m
        r = min(ranks[k + 1], m)
        ks = min(r + ks_extra, m, cols)
        if min(m, cols) <= r + ks_extra:
            total += 2.0 * m * m * cols + 2.0 * m * r * cols
        else:
            total += 2.0 * m * cols * ks * (2 + 2 * p)
        size = r * cols
        r_prev = r
    return total
