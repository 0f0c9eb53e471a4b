"""End-to-end parity of the CUDA TT-SVD / TR-SVD chain against the FP64 oracle.

Bar (from the project's correctness statement): reconstruction error within 1e-3 absolute
of the oracle's exact truncated SVD chain at the same ranks, leading singular values of
every unfolding within 1e-4 relative.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ERR_ABS = 1e-3
SIG_REL = 1e-4
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


def _to_dev(x, dev):
    import torch
    return torch.from_numpy(np.asfortranarray(x, dtype=np.float32)).to(dev)


def _cores_np(res):
    return [c.detach().cpu().numpy().astype(np.float64) for c in res.cores]


def _targets(ranks, ring):
    """Target rank of each unfolding: r0*r1 for a ring's first split, r_{k+1} otherwise."""
    d = len(ranks) - 1
    return [ranks[0] * ranks[1] if (ring and k == 0) else ranks[k + 1] for k in range(d - 1)]


# Absolute floor of the singular-value comparison, relative to sigma_1 of the unfolding:
# FP32 inputs resolve ~1e-6 of sigma_1; TF32 tensor-core operands (10-bit mantissa, rounded
# to nearest) resolve ~2e-4 of sigma_1 on unfoldings with few rows.
SIG_FLOOR = {"fp32": 2e-6, "auto": 2e-6, "tc": 2e-4}


def _check(x, res, ref_cores, ref_sig, ring, ranks, nsig=4, err_abs=ERR_ABS, sig_rel=SIG_REL,
           skip_first=False, gemm="auto"):
    """Reconstruction error within err_abs of the oracle's; leading singular values (up to the
    unfolding's target rank) within sig_rel plus the engine's floor SIG_FLOOR * sigma_1."""
    full = oracle.tr_full if ring else oracle.tt_full
    err = oracle.rel_error(x, full(_cores_np(res), "gpu"))
    err_ref = oracle.rel_error(x, full(ref_cores, "gpu"))
    assert abs(err - err_ref) <= err_abs, (err, err_ref)
    tg = _targets(ranks, ring)
    for k, s_ref in enumerate(ref_sig):
        if skip_first and k == 0:
            continue
        s = res.sigmas[k]
        kk = min(nsig, len(s), len(s_ref), tg[k])
        np.testing.assert_allclose(s[:kk], s_ref[:kk], rtol=sig_rel, atol=SIG_FLOOR[gemm] * s_ref[0],
                                   err_msg=f"unfolding {k + 1}")
    return err, err_ref


TT_CASES = [
    # (shape, ranks, noise, gemm, opts)
    ((64, 64, 64), (1, 16, 16, 1), 1e-3, "fp32", {}),
    ((64, 64, 64), (1, 16, 16, 1), 1e-3, "tc", {}),
    ((256, 256, 256), (1, 16, 16, 1), 1e-3, "fp32", {"oversample": 8, "power_iters": 1}),
    ((256, 256, 256), (1, 16, 16, 1), 1e-3, "tc", {"oversample": 8, "power_iters": 1}),
    ((256, 256, 256), (1, 16, 16, 1), 1e-3, "tc", {"oversample": 8, "power_iters": 0}),
    ((8, 8, 8, 8, 8, 8), (1, 4, 4, 4, 4, 4, 1), 1e-4, "fp32", {}),
    ((8, 8, 8, 8, 8, 8), (1, 4, 4, 4, 4, 4, 1), 1e-4, "tc", {}),
    ((12, 12, 12, 12, 12, 12), (1, 12, 20, 20, 12, 1, 1)[:7], 1e-4, "tc", {}),
    ((7, 9, 5, 8, 6), (1, 5, 9, 7, 4, 1), 1e-3, "fp32", {}),
    ((16, 16, 16, 16, 16), (1, 16, 40, 40, 16, 1), 1e-4, "tc", {}),
]


@pytest.mark.parametrize("shape,ranks,noise,gemm,opts", TT_CASES)
def test_tt_parity(gpu, shape, ranks, noise, gemm, opts):
    ttr = _ttr()
    ranks = list(ranks)
    ranks[-1] = 1
    gen_ranks = [1] + [max(1, r) for r in ranks[1:-1]] + [1]
    x = oracle.make_tt_tensor(list(shape), gen_ranks, noise, seed=11).astype(np.float64)
    res = ttr.tt_svd(_to_dev(x, gpu), ranks, gemm=gemm, **opts)
    ref_cores, ref_sig = oracle.tt_svd(x, ranks)
    for k, c in enumerate(res.cores):
        assert tuple(c.shape) == (ranks[k], shape[k], ranks[k + 1])
    _check(x, res, ref_cores, ref_sig, ring=False, ranks=ranks, gemm=gemm)


@pytest.mark.parametrize("gemm", ["fp32", "tc", "auto"])
@pytest.mark.parametrize("shape,ranks", [
    ((6, 6, 6, 6, 6, 6), (2, 3, 6, 6, 6, 3, 2)),
    ((8, 8, 8, 8, 8, 8), (2, 4, 8, 8, 8, 8, 2)),
    ((16, 16, 16, 16, 16, 16), (4, 4, 16, 16, 16, 16, 4)),
    ((40, 30, 20), (2, 10, 12, 2)),
])
def test_tr_parity(gpu, gemm, shape, ranks):
    ttr = _ttr()
    x = oracle.make_tr_tensor(list(shape), 2, 1e-4, seed=13).astype(np.float64)
    res = ttr.tr_svd(_to_dev(x, gpu), list(ranks), gemm=gemm)
    ref_cores, ref_sig = oracle.tr_svd(x, list(ranks))
    _check(x, res, ref_cores, ref_sig, ring=True, ranks=list(ranks), gemm=gemm)


@pytest.mark.parametrize("shape,gemm", [
    # unfoldings 2-4: exact 128-row steps refined by Rayleigh-Ritz on the tensor cores, the span
    # they refine taken from the subspace eigen-solver
    ((32, 32, 16, 16, 16, 8), "tc"),
    # unfolding 3: a 256-row randomized step with an 80-wide sketch (leading eigenpairs of its
    # B B^T from the subspace eigen-solver); unfolding 4: an exact 128-row refined step
    ((32, 16, 32, 16, 16, 8), "tc"),
])
def test_tr_wide_sketch_leading_eigenpairs(gpu, shape, gemm):
    """The configuration of the 32^6 ring (bond ranks 8, first split 64, oversampling 72, one
    power iteration) at smaller sizes: every later unfolding keeps 8 of up to 64 significant
    components, from eigen-solves of 80- and 128-wide Grams."""
    ttr = _ttr()
    x = oracle.make_tr_tensor(list(shape), 8, 1e-4, seed=19).astype(np.float64)
    ranks = [8] * 7
    res = ttr.tr_svd(_to_dev(x, gpu), ranks, gemm=gemm, oversample=72, power_iters=1)
    ref_cores, ref_sig = oracle.tr_svd(x, ranks)
    _check(x, res, ref_cores, ref_sig, ring=True, ranks=ranks, nsig=8, gemm=gemm)


def test_tr_rank_above_first_mode_is_zero_padded(gpu):
    # c3's first split: r0*r1 = 64 > n1 = 32 (scaled down: 4*4 = 16 > n1 = 8)
    ttr = _ttr()
    x = oracle.make_tr_tensor([8, 8, 8, 8, 8, 8], 4, 1e-4, seed=17).astype(np.float64)
    ranks = [4, 4, 4, 4, 4, 4, 4]
    res = ttr.tr_svd(_to_dev(x, gpu), ranks, gemm="tc")
    ref_cores, ref_sig = oracle.tr_svd(x, ranks)
    _check(x, res, ref_cores, ref_sig, ring=True, ranks=ranks, gemm="tc")
    g1 = res.cores[0].cpu().numpy()
    # bond components 8..15 of (a + 4 b) are zero columns
    flat = g1.transpose(1, 0, 2).reshape(8, 16, order="F")
    assert np.abs(flat[:, 8:]).max() == 0.0


@pytest.mark.parametrize("flags", ["none", "no_fold", "identity"])
def test_fold_modes_same_error(gpu, flags):
    ttr = _ttr()
    shape, ranks = (8, 8, 8, 8, 8, 8), [1, 8, 20, 20, 8, 4, 1]
    x = oracle.make_tt_tensor(list(shape), [1, 8, 8, 8, 8, 4, 1], 1e-4, seed=19).astype(np.float64)
    fl = {"none": 0, "no_fold": ttr.TT_FLAG_NO_FOLD, "identity": ttr.TT_FLAG_IDENTITY_GAUGE}[flags]
    res = ttr.tt_svd(_to_dev(x, gpu), ranks, gemm="tc", flags=fl)
    ref_cores, ref_sig = oracle.tt_svd(x, ranks)
    _check(x, res, ref_cores, ref_sig, ring=False, ranks=ranks, skip_first=(flags == "identity"), gemm="tc")
    # left-orthonormal cores (all but the last)
    for c in _cores_np(res)[:-1]:
        u = c.reshape(-1, c.shape[2], order="F")
        assert np.linalg.norm(u.T @ u - np.eye(u.shape[1])) < 1e-4


def test_golden_python_reference_through_gpu(gpu):
    """The reference's own Python TT-SVD results (golden vectors) reproduced by the CUDA chain."""
    ttr = _ttr()
    g = np.load(os.path.join(GOLD, "tt6_python_ref.npz"))
    x = g["x"]
    k = [int(v) for v in g["k"]]
    res = ttr.tt_svd(_to_dev(x, gpu), k)
    err = oracle.rel_error(x, oracle.tt_full(_cores_np(res), "gpu"))
    assert abs(err - float(g["err"])) < ERR_ABS
    for j in range(5):
        s_ref = g[f"sigma{j + 1}"]
        kk = min(3, len(res.sigmas[j]), k[j + 1])
        np.testing.assert_allclose(res.sigmas[j][:kk], s_ref[:kk], rtol=SIG_REL, atol=2e-6 * s_ref[0])


def test_golden_python_reference_tr_error(gpu):
    ttr = _ttr()
    g = np.load(os.path.join(GOLD, "tr6_python_ref_noisy.npz"))
    x = g["x"]
    k = [int(v) for v in g["k"]]
    res = ttr.tr_svd(_to_dev(x, gpu), k, gemm="tc")
    # step-1 singular values are convention independent
    np.testing.assert_allclose(res.sigmas[0][:4], g["sigma1"][:4], rtol=SIG_REL)
    err = oracle.rel_error(x, oracle.tr_full(_cores_np(res), "gpu"))
    ref_cores, _ = oracle.tr_svd(x, k, convention="gpu")
    assert abs(err - oracle.rel_error(x, oracle.tr_full(ref_cores, "gpu"))) < ERR_ABS


def test_host_io_path_and_device_error(gpu):
    ttr = _ttr()
    x = oracle.make_tt_tensor([20, 30, 40], [1, 6, 6, 1], 1e-3, seed=23)
    res = ttr.tt_svd(x, [1, 6, 6, 1])  # NumPy in, NumPy cores out
    e_host = oracle.rel_error(x, oracle.tt_full([c.astype(np.float64) for c in res.cores], "gpu"))
    import torch
    xd = _to_dev(x, gpu)
    cores = [torch.from_numpy(np.ascontiguousarray(c.transpose(2, 1, 0))).to(gpu).permute(2, 1, 0)
             for c in res.cores]
    e_dev = ttr.rel_error(xd, cores)
    assert abs(e_host - e_dev) < 1e-6
    assert e_dev < 5e-3


def test_nonfinite_input_rejected(gpu):
    ttr = _ttr()
    x = oracle.make_tt_tensor([10, 10, 10], [1, 3, 3, 1], 0.0, seed=1)
    x[3, 4, 5] = np.nan
    with pytest.raises(ttr.TTError) as e:
        ttr.tt_svd(_to_dev(x, gpu), [1, 3, 3, 1], flags=ttr.TT_FLAG_CHECK_FINITE)
    assert e.value.code == 4


@pytest.mark.parametrize("ranks", [[2, 3, 3, 1], [1, 0, 3, 1], [1, 3, 3, 2]])
def test_bad_ranks_rejected(gpu, ranks):
    ttr = _ttr()
    x = oracle.make_tt_tensor([10, 10, 10], [1, 3, 3, 1], 0.0, seed=1)
    with pytest.raises(ttr.TTError) as e:
        ttr.tt_svd(_to_dev(x, gpu), ranks)
    assert e.value.code == 3


def test_reference_entry_points(gpu, capfd):
    ttr = _ttr()
    x = oracle.make_tt_tensor([64, 64, 64], [1, 8, 8, 1], 1e-4, seed=29)
    err = np.zeros(1, np.float32)
    cr = np.zeros(1, np.float32)
    t = ttr.ttdec_gpu_float(x, [64, 64, 64], [1, 8, 8, 1], None, err, cr)
    assert t > 0 and err[0] < 1e-3
    x6 = oracle.make_tt_tensor([6] * 6, [1, 3, 3, 3, 3, 3, 1], 1e-4, seed=31)
    t6 = ttr.ttdec_half_lu_device_6(x6, [1, 3, 3, 3, 3, 3, 1], [6] * 6, 2, 64, True)
    assert t6 > 0
    out = capfd.readouterr().out
    assert "MSE:" in out
    th = ttr.ttdec_half_lu_host_6(x6, [1, 3, 3, 3, 3, 3, 1], [6] * 6, 1, 7, True)
    assert th > 0
    mse = [float(line.split("MSE:")[1].split()[0]) for line in capfd.readouterr().out.splitlines()
           if "MSE:" in line]
    assert mse and mse[-1] < 1e-3
    xr = oracle.make_tr_tensor([6] * 6, 2, 1e-4, seed=37)
    tr = ttr.trdec_half_lu_device_6(xr, [2, 2, 4, 4, 4, 4, 2], [6] * 6, 1, 64, False)
    assert tr > 0
    e3 = np.zeros(1, np.float32)
    xr3 = oracle.make_tr_tensor([30, 30, 30], 2, 1e-4, seed=41)
    t3 = ttr.trdec_gpu_float(xr3, [30, 30, 30], [2, 2, 8, 2], None, e3, None)
    assert t3 > 0 and np.isfinite(e3[0])


def test_engines_agree_and_deterministic(gpu):
    ttr = _ttr()
    x = oracle.make_tt_tensor([32, 32, 32, 32], [1, 16, 16, 16, 1], 1e-4, seed=43)
    xd = _to_dev(x, gpu)
    a = ttr.tt_svd(xd, [1, 16, 16, 16, 1], gemm="tc", seed=5)
    b = ttr.tt_svd(xd, [1, 16, 16, 16, 1], gemm="tc", seed=5)
    for ca, cb in zip(a.cores, b.cores):
        assert np.array_equal(ca.cpu().numpy(), cb.cpu().numpy())
    c = ttr.tt_svd(xd, [1, 16, 16, 16, 1], gemm="fp32", seed=5)
    ea = ttr.rel_error(xd, a.cores)
    ec = ttr.rel_error(xd, c.cores)
    # TF32 operands (round to nearest) add ~1e-4-level white error per projected step
    assert ea < ERR_ABS and ec < ERR_ABS and abs(ea - ec) < 5e-4


@pytest.mark.parametrize("gemm", ["fp32", "auto"])
@pytest.mark.parametrize("shape,ranks,noise,eps", [
    ([16, 12, 10, 14], [1, 4, 6, 3, 1], 1e-5, 1e-3),
    ([8, 9, 10, 11, 12], [1, 3, 5, 5, 4, 1], 1e-5, 1e-3),
    ([32, 32, 32, 32], [1, 8, 16, 8, 1], 1e-3, 0.02),
])
def test_adaptive_eps_matches_oracle(gpu, gemm, shape, ranks, noise, eps):
    """eps > 0: the ranks chosen by delta-truncation equal the oracle's and the error is <= eps."""
    ttr = _ttr()
    import torch
    x = oracle.make_tt_tensor(shape, ranks, noise, seed=21)
    xt = torch.from_numpy(np.ascontiguousarray(x.ravel(order="F"))).to(gpu)
    maxr = [1] + [64] * (len(shape) - 1) + [1]
    res = ttr.tt_svd(xt, maxr, gemm=gemm, eps=eps, shape=list(shape))
    ocores, oranks = oracle.tt_svd_eps(x.astype(np.float64), eps, max_ranks=maxr)
    assert res.ranks == oranks
    cores = [c.double().cpu().numpy() for c in res.cores]
    err = oracle.rel_error(x, oracle.tt_full(cores))
    assert err <= eps * 1.001
    # the estimate is the discarded energy carried in FP32 data: it can round down to 0
    assert 0.0 <= res.est_rel_err <= eps * 1.001


def test_adaptive_eps_rejects_ring(gpu):
    ttr = _ttr()
    import torch
    x = torch.randn(8 * 8 * 8, device=gpu)
    with pytest.raises(Exception):
        ttr.tr_svd(x, [2, 2, 2, 2], eps=1e-2, shape=[8, 8, 8])


@pytest.mark.parametrize("chunk", [4096, 1 << 20])
def test_host_stream_matches_device_chain(gpu, chunk):
    """TT_FLAG_HOST_STREAM: the first unfolding streamed from host memory in column chunks
    (many chunks at 4 KiB) gives the same singular values and error as the chain on a
    device-resident copy, against the oracle's exact chain."""
    import torch
    ttr = _ttr()
    shape, ranks = [16, 12, 10, 8], [1, 8, 8, 6, 1]
    x = oracle.make_tt_tensor(shape, ranks, 1e-3, seed=61)
    pinned = torch.empty(x.size, dtype=torch.float32).pin_memory()
    xs = pinned.numpy().reshape(shape[::-1]).transpose()  # Fortran-ordered view of pinned memory
    xs[...] = x
    ttr.set_stream_chunk(chunk)
    try:
        res_s = ttr.tt_svd(xs, ranks, gemm="fp32", stream=True)
    finally:
        ttr.set_stream_chunk(256 << 20)
    res_d = ttr.tt_svd(torch.from_numpy(np.ascontiguousarray(x)).to(gpu), ranks, gemm="fp32")
    err_s = oracle.rel_error(x, oracle.tt_full([np.asarray(c, dtype=np.float64) for c in res_s.cores]))
    err_d = oracle.rel_error(x, oracle.tt_full([c.double().cpu().numpy() for c in res_d.cores]))
    ocores, _ = oracle.tt_svd(x.astype(np.float64), ranks, method="gram")
    oerr = oracle.rel_error(x, oracle.tt_full(ocores))
    assert abs(err_s - err_d) < 1e-6 and abs(err_s - oerr) < 1e-3
    # the kept singular values (the rest sit at the 1e-3 noise floor, where the FP32 Gram's
    # summation order - per chunk vs whole - shows)
    for k, (a, b) in enumerate(zip(res_s.sigmas, res_d.sigmas)):
        keep = ranks[k + 1]
        np.testing.assert_allclose(a[:keep], b[:keep], rtol=1e-4)


def test_host_stream_rejects_unsupported(gpu):
    ttr = _ttr()
    x = oracle.make_tt_tensor([8, 8, 8], [1, 4, 4, 1], 1e-3, seed=2)
    with pytest.raises(ttr.TTError):
        ttr.tt_svd(x, [1, 4, 4, 1], eps=1e-2, stream=True)
    with pytest.raises(ttr.TTError):
        ttr.tr_svd(x, [2, 2, 2, 2], stream=True)
    big = np.ones((200, 4, 4), dtype=np.float32)  # first unfolding 200 x 16: randomized step
    with pytest.raises(ttr.TTError):
        ttr.tt_svd(big, [1, 4, 4, 1], stream=True)


@pytest.mark.parametrize("gemm", ["fp32", "auto"])
def test_adaptive_eps_reports_unmet_tolerance(gpu, gemm):
    """A rank bound below the eps-rank: the call says so (eps_unmet, est_rel_err > eps) instead
    of a silent success, and TT_FLAG_STRICT_EPS turns it into TT_ERR_RANK."""
    ttr = _ttr()
    import torch
    shape = [16, 12, 10, 14]
    x = oracle.make_tt_tensor(shape, [1, 6, 8, 5, 1], 1e-5, seed=23)
    xt = torch.from_numpy(np.ascontiguousarray(x.ravel(order="F"))).to(gpu)
    ok = ttr.tt_svd(xt, [1, 16, 16, 16, 1], gemm=gemm, eps=1e-3, shape=shape)
    assert ok.eps_unmet == 0 and ok.est_rel_err <= 1e-3 * 1.001
    low = ttr.tt_svd(xt, [1, 3, 3, 3, 1], gemm=gemm, eps=1e-3, shape=shape)
    assert low.eps_unmet > 0 and low.est_rel_err > 1e-3
    with pytest.raises(ttr.TTError) as ei:
        ttr.tt_svd(xt, [1, 3, 3, 3, 1], gemm=gemm, eps=1e-3, shape=shape, flags=ttr.TT_FLAG_STRICT_EPS)
    assert ei.value.code == 3  # TT_ERR_RANK


def test_unfolding1_all_sigma_full_rank(gpu):
    """A 32-row first unfolding kept at full rank (the 32^6 bench's step 1, scaled to 32^4 x 16):
    all 32 singular values within 1e-4 of the oracle's (the exact FP32-product Gram)."""
    ttr = _ttr()
    shape, ranks = [32, 32, 32, 32, 16], [1, 32, 32, 32, 16, 1]
    x = oracle.make_tt_tensor(shape, ranks, 1e-4, seed=71).astype(np.float64)
    res = ttr.tt_svd(_to_dev(x, gpu), ranks, gemm="auto", flags=ttr.TT_FLAG_KEEP_SIGMA)
    ref_cores, ref_sig = oracle.tt_svd(x, ranks)
    s, s_ref = np.asarray(res.sigmas[0], dtype=np.float64), np.asarray(ref_sig[0], dtype=np.float64)
    assert len(s) >= 32
    np.testing.assert_allclose(s[:32], s_ref[:32], rtol=1e-4, atol=SIG_FLOOR["auto"] * s_ref[0])
    _check(x, res, ref_cores, ref_sig, ring=False, ranks=ranks)


@pytest.mark.parametrize("ring,shape,ranks,s,p,gemm", [
    # TT: full-rank fold of unfolding 1, tensor-core randomized steps, exact small steps
    (False, [32, 32, 32, 16, 16, 16], [1, 32, 32, 32, 16, 16, 1], 8, 0, "auto"),
    # TR: bond split with row compaction; at s = 72 the 128-row unfolding 2 is an exact step
    # refined by Rayleigh-Ritz on the tensor-core engine, and projected plainly on FP32
    (True, [32, 32, 16, 16, 16, 16], [8] * 7, 72, 1, "auto"),
    (True, [32, 32, 16, 16, 16, 16], [8] * 7, 72, 1, "fp32"),
    (True, [32, 32, 16, 16, 16, 16], [8] * 7, 72, 1, "tc"),
    # order 3, plain FP32 EDrSVD with a power iteration (the 256^3 workload's form)
    (False, [128, 128, 128], [1, 16, 16, 1], 8, 1, "fp32"),
])
def test_bench_flop_model_matches_library(gpu, ring, shape, ranks, s, p, gemm):
    """The TFLOP/s numerator of bench.py (chain_flops, a host mirror of the plan) equals the
    arithmetic the library's pass accounting reports for the same fixed-rank chain."""
    import torch
    import bench
    ttr = _ttr()
    x = torch.randn(int(np.prod(shape)), device=gpu, dtype=torch.float32)
    fn = ttr.tr_svd if ring else ttr.tt_svd
    res = fn(x, ranks, shape=shape, gemm=gemm, oversample=s, power_iters=p)
    torch.cuda.synchronize()
    model = bench.chain_flops(shape, ranks, ring, s, p, gemm)
    assert res.flops > 0
    assert abs(model - res.flops) <= 1e-9 * res.flops, (model, res.flops)
