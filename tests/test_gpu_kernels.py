"""Kernel-level checks of libttrsvd.so on the GPU against NumPy / the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


def _randn_cm(rows, cols, seed, dev):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    a = torch.randn((cols, rows), generator=g, dtype=torch.float32)
    return a.to(dev).t()  # column-major (rows x cols)


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def test_gaussian_matches_oracle(gpu):
    ttr = _ttr()
    g = ttr.gaussian(1001, 7, seed=99, stream_id=3).cpu().numpy()
    ref = oracle.gaussian_from_philox(1001, 7, 99, 3)
    np.testing.assert_allclose(g, ref, rtol=1e-4, atol=2e-5)


# TF32 tensor cores keep 10 mantissa bits: relative error of a product-sum is ~1e-3 worst case.
TOL = {"fp32": 2e-6, "tc": 3e-3}


@pytest.mark.parametrize("gemm", ["fp32", "tc"])
@pytest.mark.parametrize("m,n,N", [(256, 4096, 24), (1024, 3000, 40), (300, 777, 17), (128, 65536, 48),
                                   (32, 5000, 32), (4096, 256, 24)])
def test_sketch(gpu, gemm, m, n, N):
    ttr = _ttr()
    a = _randn_cm(m, n, 1, gpu)
    w = _randn_cm(n, N, 2, gpu)
    y = ttr.sketch(a, w, gemm).cpu().numpy()
    ref = a.double().cpu().numpy() @ w.double().cpu().numpy()
    err = _rel(y, ref)
    assert err < TOL[gemm]
    if gemm == "tc" and m % 32 == 0 and n % 4 == 0:
        assert err > 1e-6, "TF32 rounding not visible: the tensor-core kernel did not run"


@pytest.mark.parametrize("gemm", ["fp32", "tc"])
# m <= 64 takes the one-column-per-thread kernel; small n with m >= 256 splits K.
@pytest.mark.parametrize("m,n,N", [(256, 4096, 24), (1024, 3000, 40), (32, 100000, 32), (300, 777, 17),
                                   (40, 65536, 32), (1024, 1024, 64), (37, 5000, 20), (6, 1001, 5),
                                   (64, 3001, 64), (4096, 100, 8)])
def test_project(gpu, gemm, m, n, N):
    ttr = _ttr()
    a = _randn_cm(m, n, 3, gpu)
    q = _randn_cm(m, N, 4, gpu)
    out = ttr.project(a, q, gemm).cpu().numpy()  # (N x n)
    ref = q.double().cpu().numpy().T @ a.double().cpu().numpy()
    err = _rel(out, ref)
    assert err < TOL[gemm]
    if gemm == "tc" and m % 4 == 0:
        assert err > 1e-6, "TF32 rounding not visible: the tensor-core kernel did not run"


@pytest.mark.parametrize("gemm", ["fp32", "tc"])
@pytest.mark.parametrize("m,n", [(32, 100000), (16, 5000), (48, 7777), (64, 4096), (128, 3000), (5, 999),
                                 (32, 4096 * 37 + 12), (20, 50001), (36, 12345), (40, 300000), (64, 20000),
                                 (33, 9000)])
def test_gram_rows(gpu, gemm, m, n):
    ttr = _ttr()
    a = _randn_cm(m, n, 5, gpu)
    w = ttr.gram_rows(a, gemm).cpu().numpy()
    ad = a.double().cpu().numpy()
    # TF32 rounding (RMS ~2.8e-4 per product) of independent columns averages out in the
    # sum over n; relative to ||W||_F the error is ~2.8e-4 * sqrt(m / n).  The tensor cores'
    # FP32 accumulation truncates, which shrinks the positive diagonal sums by up to ~2e-5
    # relative however long n is.
    tol = 1e-6 if gemm == "fp32" else 6e-4 * np.sqrt(m / n) + 2e-5
    assert _rel(w, ad @ ad.T) < tol


@pytest.mark.parametrize("m,n", [(32, 65536), (40, 4096), (128, 1024)])
def test_gram_rows_tc_runs_on_tensor_cores(gpu, m, n):
    """1 + 2^-12 is not representable in TF32 and rounds to 1 on the tensor-core path."""
    import torch
    ttr = _ttr()
    a = torch.full((n, m), 1.0 + 2.0 ** -12, device=gpu).t()
    w = ttr.gram_rows(a, "tc").cpu().numpy()
    np.testing.assert_allclose(w, np.full((m, m), float(n)), rtol=1e-6)


@pytest.mark.parametrize("n,N", [(100000, 40), (5000, 16), (777, 48), (4096, 64), (3000, 128), (50000, 24),
                                 (8192, 64), (65537, 33), (1 << 20, 48)])
def test_gram_tall(gpu, n, N):
    ttr = _ttr()
    z = _randn_cm(n, N, 6, gpu)
    w = ttr.gram_tall(z).cpu().numpy()
    zd = z.double().cpu().numpy()
    assert _rel(w, zd.T @ zd) < 1e-12


@pytest.mark.parametrize("n,N", [(100000, 40), (9000, 24), (65536 + 7, 64), (20000, 32), (50000, 44)])
def test_gram_tall_rowmajor(gpu, n, N):
    """Contiguous rows (the projected factor's layout): FP64 accumulation of every product."""
    import torch
    ttr = _ttr()
    g = torch.Generator(device="cpu").manual_seed(7)
    z = torch.randn(n, N, generator=g).to(gpu)
    w = ttr.gram_tall(z, rowmajor=True).cpu().numpy()
    zd = z.double().cpu().numpy()
    assert _rel(w, zd.T @ zd) < 1e-12


# (1024, 40), (512, 64), (1000, 33), (64, 5), (7, 3), (2048, 16), (1024, 48), (4096, 16) take the
# single-launch kernel (a cluster of up to 8 CTAs, >= 128 rows each, in shared memory: 1, 4 and 8
# CTAs among these); the others take the multi-kernel path.
@pytest.mark.parametrize("n,N", [(1024, 40), (512, 64), (1000, 33), (64, 5), (7, 3), (2048, 16), (1024, 48),
                                 (100000, 24), (5000, 64), (300, 128), (4096, 16)])
def test_cholqr2(gpu, n, N):
    ttr = _ttr()
    y = _randn_cm(n, N, 7, gpu)
    q, r = ttr.cholqr2(y)
    qd = q.double().cpu().numpy()
    rd = r.cpu().numpy()
    orth = np.linalg.norm(qd.T @ qd - np.eye(N))
    assert orth < 1e-5
    assert _rel(qd @ rd, y.double().cpu().numpy()) < 1e-5


@pytest.mark.parametrize("n,N", [(256, 65), (256, 80), (462, 72), (462, 80), (463, 80), (2000, 80), (5000, 64)])
def test_cholqr2_without_r(gpu, n, N):
    """The decomposition's form (no R): up to 80 columns and ~460 rows in one CTA, larger sketches
    through the cluster or the multi-launch path; Q orthonormal and spanning Y."""
    ttr = _ttr()
    y = _randn_cm(n, N, 11, gpu)
    q, r = ttr.cholqr2(y, want_r=False)
    assert r is None
    qd = q.double().cpu().numpy()
    yd = y.double().cpu().numpy()
    assert np.linalg.norm(qd.T @ qd - np.eye(N)) < 1e-5
    assert _rel(qd @ (qd.T @ yd), yd) < 1e-5


def test_cholqr2_rank_deficient_zeroes_dependent_columns(gpu):
    import torch
    ttr = _ttr()
    base = _randn_cm(2000, 6, 8, gpu)
    y = torch.cat([base, base[:, :2] * 2.0], dim=1)
    y = y.t().contiguous().t()
    q, _ = ttr.cholqr2(y)
    qd = q.double().cpu().numpy()
    norms = np.linalg.norm(qd, axis=0)
    assert np.all(norms[:6] > 0.99) and np.all(norms[6:] < 1e-3)


@pytest.mark.parametrize("N", [1, 2, 5, 24, 31, 32, 33, 40, 44, 45, 46, 47, 63, 64, 65, 96, 128])
def test_syev(gpu, N):
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(N)
    b = rng.standard_normal((N, N + 7))
    w = b @ b.T
    ev, vec, sweeps = ttr.syev(torch.from_numpy(w).to(gpu))
    ev = ev.cpu().numpy()
    vec = vec.cpu().numpy()
    ref = np.sort(np.linalg.eigvalsh(w))[::-1]
    np.testing.assert_allclose(ev, ref, rtol=1e-11, atol=1e-11 * ref[0])
    assert np.linalg.norm(w @ vec - vec * ev) < 1e-10 * ref[0] * N
    assert np.linalg.norm(vec.T @ vec - np.eye(N)) < 1e-12 * N
    assert 1 <= sweeps <= 40


@pytest.mark.parametrize("N,rank", [(40, 12), (64, 1), (32, 0), (96, 30)])
def test_syev_rank_deficient_terminates(gpu, N, rank):
    """Gram matrices of rank-deficient sketches have eigenvalues at the FP64 rounding floor;
    the sweep loop must still converge (rotations below that floor are skipped)."""
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(N + rank)
    b = rng.standard_normal((N, rank))
    w = b @ b.T
    ev, vec, sweeps = ttr.syev(torch.from_numpy(w).to(gpu))
    ev = ev.cpu().numpy()
    vec = vec.cpu().numpy()
    ref = np.sort(np.linalg.eigvalsh(w))[::-1]
    scale = max(ref[0], 1.0)
    np.testing.assert_allclose(ev, ref, atol=1e-12 * scale * N)
    assert np.linalg.norm(vec.T @ vec - np.eye(N)) < 1e-12 * N
    assert 1 <= sweeps < 40


@pytest.mark.parametrize("N", [16, 40, 96])
def test_syev_asymmetric_rounding_converges(gpu, N):
    """Tensor-core Grams are symmetric only to FP32 rounding; the solver symmetrises its input
    and must converge to the eigen-decomposition of (W + W^T) / 2."""
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(N)
    b = rng.standard_normal((N, 3 * N))
    w = b @ b.T
    w_in = w + 1e-7 * np.abs(w).max() * np.triu(rng.standard_normal((N, N)), 1)
    ev, vec, sweeps = ttr.syev(torch.from_numpy(w_in).to(gpu))
    ev = ev.cpu().numpy()
    vec = vec.cpu().numpy()
    ws = 0.5 * (w_in + w_in.T)
    ref = np.sort(np.linalg.eigvalsh(ws))[::-1]
    np.testing.assert_allclose(ev, ref, rtol=1e-11, atol=1e-11 * ref[0])
    assert np.linalg.norm(ws @ vec - vec * ev) < 1e-10 * ref[0] * N
    assert sweeps < 20


@pytest.mark.parametrize("N", [3, 16, 31])
def test_syev_warp_sizes_and_clusters(gpu, N):
    """N <= 32 runs the one-warp register-resident solver; clustered (repeated) eigenvalues."""
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(100 + N)
    q, _ = np.linalg.qr(rng.standard_normal((N, N)))
    lam = np.repeat(np.array([3.0, 1.0, 1e-3, 0.0]), (N + 3) // 4)[:N]
    w = (q * lam) @ q.T
    ev, vec, sweeps = ttr.syev(torch.from_numpy(w).to(gpu))
    ev = ev.cpu().numpy()
    vec = vec.cpu().numpy()
    np.testing.assert_allclose(ev, np.sort(lam)[::-1], atol=1e-12)
    assert np.linalg.norm(w @ vec - vec * ev) < 1e-12 * N
    assert np.linalg.norm(vec.T @ vec - np.eye(N)) < 1e-12 * N
    assert 1 <= sweeps < 40


@pytest.mark.parametrize("N", [20, 32, 40])
def test_syev_graded_spectrum_relative_accuracy(gpu, N):
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(1)
    q, _ = np.linalg.qr(rng.standard_normal((N, N)))
    lam = np.logspace(0, -10, N)
    w = (q * lam) @ q.T
    ev, _, _ = ttr.syev(torch.from_numpy(w).to(gpu))
    keep = lam >= 1e-6  # FP64 rounding of W (1e-16 absolute) leaves 1e-10 relative there
    np.testing.assert_allclose(ev.cpu().numpy()[keep], lam[keep], rtol=1e-8)


@pytest.mark.parametrize("r0,r1,n", [(8, 8, 100000), (2, 4, 777), (1, 32, 5000), (3, 5, 12345)])
def test_permute231_bit_exact(gpu, r0, r1, n):
    import torch
    ttr = _ttr()
    x = torch.randn(r0 * r1 * n, device=gpu)
    out = ttr.permute231(x, r0, r1, n).cpu().numpy()
    ref = x.cpu().numpy().reshape(r0, r1, n, order="F").transpose(1, 2, 0).ravel(order="F")
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("kind", ["project", "sketch"])
def test_tc_rounding_bias(gpu, kind):
    """Positive operands expose a systematic bias: truncating FP32 to TF32 toward zero shrinks
    every product by ~3e-4 on average, which would scale the projection coherently.  The
    projection must be unbiased (Q split into hi/lo parts, A converted by the TMA unit)."""
    import torch
    ttr = _ttr()
    g = torch.Generator(device="cpu").manual_seed(5)
    m, n, N = 256, 8192, 32
    a = (1.0 + torch.rand((n, m), generator=g)).to(gpu).t()
    if kind == "project":
        q = (1.0 + torch.rand((N, m), generator=g)).to(gpu).t()
        out = ttr.project(a, q, "tc").double().cpu().numpy()
        ref = q.double().cpu().numpy().T @ a.double().cpu().numpy()
    else:
        w = (1.0 + torch.rand((N, n), generator=g)).to(gpu).t()
        out = ttr.sketch(a, w, "tc").cpu().numpy()
        ref = a.double().cpu().numpy() @ w.double().cpu().numpy()
    bias = float(np.mean(out / ref - 1.0))
    print(f"{kind} relative bias {bias:.3e}")
    if kind == "project":
        assert abs(bias) < 5e-5, f"projection bias {bias:.3e}"
    else:
        assert abs(bias) < 2e-3, f"sketch bias {bias:.3e}"


@pytest.mark.parametrize("n", [1 << 21, 3 << 20])
def test_gram_rows_tc_resolves_graded_spectrum(gpu, n):
    """A 32-row unfolding with singular values from 1 down to 3e-3 (eigenvalues over 5 decades,
    like unfolding 1 of the 32^6 TT).  The tensor-core Gram accumulates in FP32 over units of
    at most 2048 columns and in FP64 across units, so the leading eigenvalues (above 1e-2 of the
    largest) stay within 1e-4 relative of the FP64 ones; the others within 2e-6 of the largest
    in absolute terms, the floor the TF32 rounding of the operand sets (the smallest, 1e-5 of
    the largest, move by up to ~5 %)."""
    import torch
    ttr = _ttr()
    m = 32
    g = torch.Generator(device="cpu").manual_seed(9)
    u, _ = torch.linalg.qr(torch.randn(m, m, generator=g, dtype=torch.float64))
    sig = torch.logspace(0, -2.5, m, dtype=torch.float64)
    z = torch.randn(n, m, generator=g, dtype=torch.float32).to(gpu)
    z = z / torch.linalg.vector_norm(z, dim=0, keepdim=True)
    a_t = (z.double() @ (u * sig).T.to(gpu)).float()  # (n x m) row-major = A (m x n) column-major
    a = a_t.t()
    w = ttr.gram_rows(a, "tc").cpu().numpy()
    ad = a_t.double().cpu().numpy()
    ref = np.sort(np.linalg.eigvalsh(ad.T @ ad))[::-1]
    got = np.sort(np.linalg.eigvalsh(0.5 * (w + w.T)))[::-1]
    lead = ref >= 1e-2 * ref[0]
    np.testing.assert_allclose(got[lead], ref[lead], rtol=1e-4)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=2e-6 * ref[0])


@pytest.mark.parametrize("gemm", ["fp32", "auto"])
@pytest.mark.parametrize("m,n", [(32, 1), (32, 47), (32, 48 * 8 * 148 + 5), (32, 1 << 20), (16, 100003),
                                 (8, 333333), (28, 70000), (4, 5000), (12, 48), (24, 4096 * 37 + 12)])
def test_gram_rows_exact_short_vectors(gpu, gemm, m, n):
    """Up to 32 rows the exact CUDA-core Gram runs (FP32 products, FP64 sums): ~1e-9 relative."""
    ttr = _ttr()
    a = _randn_cm(m, n, 15, gpu)
    w = ttr.gram_rows(a, gemm).cpu().numpy()
    ad = a.double().cpu().numpy()
    ref = ad @ ad.T
    # a handful of vectors leaves one FP32-rounded partial sum per entry (~6e-8); long inputs
    # average many of them
    assert _rel(w, ref) < (2e-7 if n < 65536 else 5e-8)
    np.testing.assert_array_equal(w, w.T)


@pytest.mark.parametrize("n", [1 << 21, 3 << 20])
def test_gram_rows_exact_resolves_graded_spectrum(gpu, n):
    """The same graded 32-row unfolding as above (eigenvalues over 5 decades, like unfolding 1
    of the 32^6 TT): the exact kernel gives every eigenvalue, the smallest at 1e-5 of the
    largest included, within 1e-4 relative (singular values within 5e-5)."""
    import torch
    ttr = _ttr()
    m = 32
    g = torch.Generator(device="cpu").manual_seed(9)
    u, _ = torch.linalg.qr(torch.randn(m, m, generator=g, dtype=torch.float64))
    sig = torch.logspace(0, -2.5, m, dtype=torch.float64)
    z = torch.randn(n, m, generator=g, dtype=torch.float32).to(gpu)
    z = z / torch.linalg.vector_norm(z, dim=0, keepdim=True)
    a_t = (z.double() @ (u * sig).T.to(gpu)).float()
    a = a_t.t()
    w = ttr.gram_rows(a, "auto").cpu().numpy()
    ad = a_t.double().cpu().numpy()
    ref = np.sort(np.linalg.eigvalsh(ad.T @ ad))[::-1]
    got = np.sort(np.linalg.eigvalsh(0.5 * (w + w.T)))[::-1]
    np.testing.assert_allclose(got, ref, rtol=1e-4)


def test_gram_rows_exact_is_deterministic(gpu):
    ttr = _ttr()
    a = _randn_cm(32, 3 << 18, 21, gpu)
    w1 = ttr.gram_rows(a, "auto").cpu().numpy()
    w2 = ttr.gram_rows(a, "auto").cpu().numpy()
    np.testing.assert_array_equal(w1, w2)
