"""The CPU oracle, pinned against the reference's own Python TR-SVD (golden vectors) and
against published known-answer vectors of Philox4x32-10."""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("name", ["tr6_python_ref.npz", "tr6_python_ref_noisy.npz"])
def test_tr_oracle_matches_reference_python(name):
    g = _load(name)
    x, k = g["x"], [int(v) for v in g["k"]]
    cores, sig = oracle.tr_svd(x, k, convention="python")
    for j in range(6):
        ref = g[f"core{j + 1}"]
        assert ref.shape == cores[j].shape
        np.testing.assert_allclose(cores[j], ref, rtol=0, atol=1e-12)
    for j in range(5):
        np.testing.assert_allclose(sig[j], g[f"sigma{j + 1}"], rtol=1e-12, atol=1e-12)
    err = oracle.rel_error(x, oracle.tr_full(cores, "python"))
    assert abs(err - float(g["err"])) < 1e-12


def test_tt_oracle_matches_reference_python():
    g = _load("tt6_python_ref.npz")
    x, k = g["x"], [int(v) for v in g["k"]]
    cores, sig = oracle.tt_svd(x, k, convention="python")
    for j in range(6):
        np.testing.assert_allclose(cores[j], g[f"core{j + 1}"], rtol=0, atol=1e-12)
    err = oracle.rel_error(x, oracle.tt_full(cores, "python"))
    assert abs(err - float(g["err"])) < 1e-12
    # the column-major (GPU) chain sees the same unfoldings up to row/column permutations
    cg, sg = oracle.tt_svd(np.asfortranarray(x), k, convention="gpu")
    for j in range(5):
        np.testing.assert_allclose(sg[j], g[f"sigma{j + 1}"], rtol=1e-10, atol=1e-12)
    assert abs(oracle.rel_error(x, oracle.tt_full(cg, "gpu")) - float(g["err"])) < 1e-10


def test_gram_method_equals_svd_method():
    x = oracle.make_tt_tensor([5, 6, 4, 5], [1, 3, 4, 2, 1], 1e-3, seed=3).astype(np.float64)
    c1, s1 = oracle.tt_svd(x, [1, 3, 4, 2, 1], method="svd")
    c2, s2 = oracle.tt_svd(x, [1, 3, 4, 2, 1], method="gram")
    e1 = oracle.rel_error(x, oracle.tt_full(c1))
    e2 = oracle.rel_error(x, oracle.tt_full(c2))
    assert abs(e1 - e2) < 1e-9
    for a, b in zip(s1, s2):
        k = min(len(a), len(b), 3)
        np.testing.assert_allclose(a[:k], b[:k], rtol=1e-9)


def test_tr_gpu_convention_exact_for_ring_input():
    # The bond split of step 1 is arbitrary, so later unfoldings of a bond-2 ring can need
    # rank r0*r1*r_k; with those ranks the chain is exact.
    x = oracle.make_tr_tensor([4, 5, 4, 3], 2, 0.0, seed=5).astype(np.float64)
    cores, _ = oracle.tr_svd(x, [2, 2, 10, 12, 2], convention="gpu")
    assert oracle.rel_error(x, oracle.tr_full(cores, "gpu")) < 1e-10


def test_zero_padding_beyond_unfolding_rank():
    x = oracle.make_tr_tensor([3, 4, 4, 3], 2, 1e-3, seed=9).astype(np.float64)
    cores, _ = oracle.tr_svd(x, [3, 2, 4, 4, 3], convention="gpu")  # r0*r1 = 6 > n1 = 3
    assert cores[0].shape == (3, 3, 2)
    err = oracle.rel_error(x, oracle.tr_full(cores, "gpu"))
    assert np.isfinite(err) and err < 1.0


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, expect):
    out = oracle.philox4x32_10(np.array([ctr], dtype=np.uint32), key)
    assert tuple(int(v) for v in out[0]) == expect


def test_gaussian_moments():
    g = oracle.gaussian_from_philox(4096, 8, seed=1234)
    assert abs(g.mean()) < 0.02 and abs(g.std() - 1) < 0.02


def test_edrsvd_restatements_recover_low_rank():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((60, 8)) @ rng.standard_normal((8, 300))
    om = rng.standard_normal((300, 12))
    u, s, vt = oracle.edrsvd_plain(a, 8, 4, 1, om)
    assert np.linalg.norm(a - (u[:, :8] * s[:8]) @ vt[:8]) / np.linalg.norm(a) < 1e-10
    u2, s2, svt = oracle.edrsvd_gram(a, 8, 4, 1, om)
    assert np.linalg.norm(a - u2[:, :8] @ svt[:8]) / np.linalg.norm(a) < 1e-8
    np.testing.assert_allclose(s[:8], s2[:8], rtol=1e-8)


def test_flops_model_c2():
    f = oracle.tt_flops_model([32] * 6, [1, 32, 32, 32, 32, 32, 1], 8, 0)
    assert f > 1e11


def test_tt_svd_eps_meets_tolerance_and_recovers_ranks():
    """delta-truncation: error <= eps and, on a noisy low-rank TT, the generating ranks."""
    x = oracle.make_tt_tensor([6, 7, 5, 8], [1, 3, 4, 2, 1], 1e-6, seed=11).astype(np.float64)
    cores, ranks = oracle.tt_svd_eps(x, 1e-3)
    assert ranks == [1, 3, 4, 2, 1]
    err = oracle.rel_error(x, oracle.tt_full(cores))
    assert err <= 1e-3
    cores, ranks = oracle.tt_svd_eps(x, 0.3)
    assert oracle.rel_error(x, oracle.tt_full(cores)) <= 0.3
    assert all(a <= b for a, b in zip(ranks, [1, 3, 4, 2, 1]))
