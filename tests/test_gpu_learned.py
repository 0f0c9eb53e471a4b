"""Learned EDrSVD predictor on the GPU: the network kernels against the CPU oracle, training,
and the predictor / plain adaptive EDrSVD inside the chain."""
import numpy as np
import pytest

import oracle
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, M.N_IN)).astype(np.float32)
    t = rng.standard_normal((n, M.N_OUT)).astype(np.float32)
    return x, t


def test_mlp_forward_matches_oracle(gpu):
    import torch
    ttr = _ttr()
    p = M.init_params(3).astype(np.float32)
    x, _ = _data(300, 1)
    y = ttr.mlp_forward(torch.from_numpy(p).to(gpu), torch.from_numpy(x).to(gpu)).cpu().numpy()
    ref, _ = M.forward(p.astype(np.float64), x.astype(np.float64))
    np.testing.assert_allclose(y, ref, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("n", [1, 8, 37, 256])
def test_mlp_grad_matches_oracle(gpu, n):
    """Backward kernel (hidden-unit-parallel groups, fixed-order sum of the group partials)
    against the oracle's backpropagation in FP64."""
    import torch
    ttr = _ttr()
    p = M.init_params(5).astype(np.float32)
    x, t = _data(n, 2)
    g, loss = ttr.mlp_grad(torch.from_numpy(p).to(gpu), torch.from_numpy(x).to(gpu), torch.from_numpy(t).to(gpu))
    lref, gref = M.loss_and_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    g = g.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - gref) <= 2e-6 * np.linalg.norm(gref) + 1e-7
    assert abs(float(loss.cpu()[0]) - lref) <= 1e-5 * lref


def _minibatch(step, batch, n, seed):
    """The training kernel's draw: sample slot b of step s is Philox word 0 of counter
    (s, b, 0x4d4c50, 0) under key = seed, modulo n."""
    ctr = np.zeros((batch, 4), dtype=np.uint32)
    ctr[:, 0] = step
    ctr[:, 1] = np.arange(batch)
    ctr[:, 2] = 0x4d4c50
    return oracle.philox4x32_10(ctr, (seed & 0xFFFFFFFF, seed >> 32))[:, 0] % n


def test_mlp_train_steps_match_oracle_adam(gpu):
    """Each Adam step of the training kernel equals the oracle's Adam applied to the kernel's
    gradient of the same minibatch (the gradient itself is checked against the oracle above);
    three steps in one persistent launch equal three one-step launches bitwise."""
    import torch
    ttr = _ttr()
    n, batch, steps, seed, lr = 50, 24, 3, 99, 1e-2
    p0 = M.init_params(7).astype(np.float32)
    x, t = _data(n, 4)
    xd, td = torch.from_numpy(x).to(gpu), torch.from_numpy(t).to(gpu)
    p = torch.from_numpy(p0).to(gpu)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    mr, vr = np.zeros(p0.size), np.zeros(p0.size)
    for step in range(steps):
        idx = _minibatch(step, batch, n, seed)
        before = p.cpu().numpy().astype(np.float64)
        g, loss = ttr.mlp_grad(p, xd[idx], td[idx])
        trace = ttr.mlp_train(p, m, v, xd, td, 1, batch=batch, lr=lr, step0=step, seed=seed).cpu().numpy()
        assert trace[0] == float(loss.cpu()[0])
        lref, gref = M.loss_and_grad(before, x[idx].astype(np.float64), t[idx].astype(np.float64))
        assert abs(trace[0] - lref) <= 1e-5 * lref
        pr, mr, vr = M.adam_step(before, g.cpu().numpy().astype(np.float64), mr, vr, step + 1, lr)
        np.testing.assert_allclose(p.cpu().numpy(), pr, rtol=0, atol=2e-6)
    p3 = torch.from_numpy(p0).to(gpu)
    m3 = torch.zeros_like(p3)
    v3 = torch.zeros_like(p3)
    ttr.mlp_train(p3, m3, v3, xd, td, steps, batch=batch, lr=lr, step0=0, seed=seed)
    assert torch.equal(p3, p) and torch.equal(m3, m) and torch.equal(v3, v)


def test_mlp_training_fits_a_smooth_map(gpu):
    import torch
    ttr = _ttr()
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (4096, M.N_IN)).astype(np.float32)
    w = rng.standard_normal((M.N_IN, M.N_OUT))
    t = np.tanh(x @ w).astype(np.float32)
    p = torch.from_numpy(M.init_params(2).astype(np.float32)).to(gpu)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    trace = ttr.mlp_train(p, m, v, torch.from_numpy(x).to(gpu), torch.from_numpy(t).to(gpu), 1500, batch=128,
                          lr=3e-3, seed=5).cpu().numpy()
    assert trace[-100:].mean() < 0.05 * trace[:20].mean()
    y = ttr.mlp_forward(p, torch.from_numpy(x).to(gpu)).cpu().numpy()
    assert np.mean(np.sum((y - t) ** 2, axis=1)) < 0.02


def test_probe_features_follow_the_spectrum(gpu):
    """Features of diag(sigma) and of U diag(sigma) V^T (orthonormal U, V) agree up to the
    probe's randomness, and the decay features order spectra by alpha."""
    import torch
    ttr = _ttr()
    k, n = 256, 4096
    g = torch.Generator().manual_seed(0)
    u, _ = torch.linalg.qr(torch.randn(k, k, generator=g, dtype=torch.float64))
    vq, _ = torch.linalg.qr(torch.randn(n, k, generator=g, dtype=torch.float64))
    feats = {}
    for alpha in (0.6, 1.2, 2.0):
        sig = torch.arange(1, k + 1, dtype=torch.float64) ** (-alpha)
        a = ((u * sig) @ vq.T).float().to(gpu)  # k x n, row-major -> column-major copy inside
        d = torch.diag(sig.float()).to(gpu)
        fa = np.mean([ttr.probe_features(a, tol=1e-3, seed=s).cpu().numpy() for s in range(8)], axis=0)
        fd = np.mean([ttr.probe_features(d, energy=float((sig ** 2).sum()), tol=1e-3, seed=100 + s).cpu().numpy()
                      for s in range(8)], axis=0)
        assert abs(fa[0] - np.log2(k) / 10) < 1e-6 and abs(fa[7] - np.log10(1e-3) / 4) < 1e-6
        np.testing.assert_allclose(fa[1:7], fd[1:7], atol=0.1)
        feats[alpha] = fa
    assert feats[2.0][3] < feats[1.2][3] < feats[0.6][3]  # log10(mu_8 / mu_1) falls with alpha


def _lowrank(m, n, alpha, seed, gpu, rank=None):
    import torch
    g = torch.Generator().manual_seed(seed)
    k = min(m, n)
    u, _ = torch.linalg.qr(torch.randn(m, k, generator=g, dtype=torch.float64))
    v, _ = torch.linalg.qr(torch.randn(n, k, generator=g, dtype=torch.float64))
    sig = torch.arange(1, k + 1, dtype=torch.float64) ** (-alpha)
    if rank is not None:
        sig[rank:] = 0.0
    a = ((u * sig) @ v.T).float()
    return a.to(gpu), sig.numpy()


def _err(ttr, a, res):
    import torch
    u = res.cores[0].reshape(res.cores[0].shape[1], -1).double()
    w = res.cores[1].reshape(res.cores[1].shape[0], -1).double()
    return float(torch.linalg.matrix_norm(a.double() - u @ w) / torch.linalg.matrix_norm(a.double()))


def test_plain_adaptive_sketch_width_grows_until_tolerance(gpu):
    ttr = _ttr()
    a, sig = _lowrank(512, 20000, 2.0, 1, gpu)
    tol = 1e-3
    res = ttr.tt_svd(a, [1, 120, 1], eps=tol, power_iters=1, flags=ttr.TT_FLAG_ADAPTIVE_KS, gemm="fp32")
    assert res.step_attempts[0] >= 2 and res.step_ks[0] <= 128
    assert res.est_rel_err <= tol
    assert _err(ttr, a, res) <= tol * 1.05
    assert res.passes == 4 * res.step_attempts[0]


def test_learned_fallback_takes_over_a_bad_prediction(gpu):
    """A predictor that always answers rank 2, oversampling 2, no power iteration: the
    a-posteriori estimate exceeds the tolerance, the plain adaptive method takes over and the
    result still meets it."""
    ttr = _ttr()
    p = np.zeros(M.N_PARAMS, dtype=np.float32)
    p[-3:] = [0.1, 0.2, 0.0]  # b3: log2 r / 10 = 0.1, log2 s / 5 = 0.2
    ttr.set_predictor(p)
    try:
        a, _ = _lowrank(512, 20000, 2.0, 2, gpu)
        tol = 1e-3
        res = ttr.tt_svd(a, [1, 120, 1], eps=tol, power_iters=1, flags=ttr.TT_FLAG_LEARNED, gemm="fp32")
        assert res.fallbacks == 1 and res.step_attempts[0] >= 2
        assert res.est_rel_err <= tol and _err(ttr, a, res) <= tol * 1.05
    finally:
        ttr.set_predictor(None)


def test_learned_flag_needs_predictor_and_eps(gpu):
    ttr = _ttr()
    a, _ = _lowrank(256, 4096, 2.0, 3, gpu)
    with pytest.raises(ttr.TTError):
        ttr.tt_svd(a, [1, 64, 1], eps=1e-3, flags=ttr.TT_FLAG_LEARNED)
    with pytest.raises(ttr.TTError):
        ttr.tt_svd(a, [1, 64, 1], eps=0.0, flags=ttr.TT_FLAG_ADAPTIVE_KS)


def test_trained_predictor_saves_passes_at_equal_error(gpu):
    """The shipped predictor (trained by the library's kernels, learned.py) against the plain
    adaptive EDrSVD on held-out power-law unfoldings U diag(i^-alpha) V^T: fewer passes over A
    in total, and per matrix the same achieved error (the tolerance, or what the 128-column
    sketch limit allows when the exact rank is above it)."""
    import torch
    ttr = _ttr()
    from tensor_train_ring_decompositions_hpc_gpu_b200 import learned
    ttr.set_predictor(learned.load_params())
    tol = 1e-3
    tot = {"plain": 0, "learned": 0}
    try:
        for i, (m, alpha) in enumerate([(300, 0.7), (600, 1.3), (300, 1.9), (600, 2.0), (450, 1.6), (600, 1.85)]):
            a, _ = _lowrank(m, 32768, alpha, 50 + i, gpu)
            errs = {}
            for name, flag in (("plain", ttr.TT_FLAG_ADAPTIVE_KS), ("learned", ttr.TT_FLAG_LEARNED)):
                res = ttr.tt_svd(a, [1, 120, 1], eps=tol, power_iters=1, flags=flag)
                errs[name] = _err(ttr, a, res)
                tot[name] += res.passes
                # the a-posteriori estimate is the achieved error
                assert abs(res.est_rel_err - errs[name]) <= 0.05 * errs[name] + 1e-5, (m, alpha, name)
            assert errs["learned"] <= max(tol, errs["plain"]) * 1.05, (m, alpha, errs)
    finally:
        ttr.set_predictor(None)
    assert tot["learned"] <= 0.6 * tot["plain"], tot
