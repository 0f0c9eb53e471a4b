"""CPU checks of the learned-predictor pieces: the oracle network's gradient against finite
differences, and the label generator against direct computation."""
import numpy as np

from oracle import mlp_oracle as M
from tensor_train_ring_decompositions_hpc_gpu_b200 import learned


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(1)
    x = rng.standard_normal((17, M.N_IN))
    t = rng.standard_normal((17, M.N_OUT))
    _, g = M.loss_and_grad(p, x, t)
    idx = rng.choice(M.N_PARAMS, 60, replace=False)
    h = 1e-6
    for q in idx:
        e = np.zeros_like(p)
        e[q] = h
        fd = (M.loss_and_grad(p + e, x, t)[0] - M.loss_and_grad(p - e, x, t)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (q, fd, g[q])


def test_oracle_adam_step_is_bias_corrected():
    p = np.ones(5)
    g = np.array([1.0, -2.0, 0.5, 0.0, 3.0])
    p1, m, v = M.adam_step(p, g, np.zeros(5), np.zeros(5), 1, lr=0.1)
    # first bias-corrected step moves every parameter with a nonzero gradient by ~lr
    np.testing.assert_allclose(p1[g != 0], p[g != 0] - 0.1 * np.sign(g[g != 0]), rtol=1e-6)
    assert p1[3] == 1.0


def test_param_layout_matches_library_constants():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    assert M.N_PARAMS == _lib.TT_MLP_PARAMS == learned.init_params(0).size
    assert M.N_IN == _lib.TT_MLP_INPUTS and M.N_OUT == _lib.TT_MLP_OUTPUTS


def test_exact_rank_and_labels():
    sig = learned.spectrum(300, 2.0)
    e = sig ** 2
    for tol in (1e-3, 3e-3):
        r = learned.exact_rank(sig, tol, cap=300)
        assert e[r:].sum() <= tol * tol * e.sum() < e[r - 1:].sum()
    # fast decay: a feasible label; a pure slow power law over 400 values: the width-limit label
    r, s, p, ok = learned.label(400, 2.0, 2e-3, seed=3)
    assert ok and r <= learned.RANK_CAP and s in learned.OVERSAMPLE and p in learned.POWER
    assert learned.label(400, 0.6, 1e-3, seed=3) == (learned.RANK_CAP, 8, 1, False)


def test_training_spectra_have_reachable_ranks():
    """Bond-limited spectra with a noise floor below tol / 4: the eps-rank stays within the bond
    (plus the floor's share), so the labels are reachable targets."""
    k, alpha, tol, bond, eta = learned.sample_specs(200, seed=11)
    assert np.all(eta <= tol / 4 * (1 + 1e-12)) and np.all(bond < k)
    for i in range(0, 200, 10):
        sig = learned.spectrum(k[i], alpha[i], bond[i], eta[i])
        e = sig ** 2
        assert abs(e[bond[i]:].sum() / e.sum() - eta[i] ** 2) < 1e-9
        assert learned.exact_rank(sig, tol[i], cap=int(k[i])) <= bond[i]
    r, s, p, ok = learned.label(int(k[0]), float(alpha[0]), float(tol[0]), 5, int(bond[0]), float(eta[0]))
    assert ok and r <= bond[0]


def test_targets_decode_round_trip():
    r = np.array([1, 7, 40, 120])
    s = np.array([4, 8, 16, 32])
    p = np.array([0, 1, 2, 1])
    rr, ss, pp, ks = learned.decode(learned.targets(r, s, p))
    np.testing.assert_array_equal(rr, r)
    np.testing.assert_array_equal(ss, s)
    np.testing.assert_array_equal(pp, p)
    np.testing.assert_array_equal(ks, np.minimum(r + s, 128))
