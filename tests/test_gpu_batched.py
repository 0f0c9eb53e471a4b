"""Batched small-tensor TT-SVD (tt_svd_batched) against the oracle's delta-truncated TT-SVD."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _ttr():
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    return ttr


def _batch(count, seed, dmin=8, dmax=32, rmin=2, rmax=16, noise=1e-3, order=4):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = [int(v) for v in rng.integers(dmin, dmax + 1, size=order)]
        r = [1] + [int(v) for v in rng.integers(rmin, rmax + 1, size=order - 1)] + [1]
        out.append(oracle.make_tt_tensor(n, r, noise, seed=int(rng.integers(1 << 30))))
    return out


@pytest.mark.parametrize("eps", [1e-2, 5e-2])
def test_batched_matches_oracle_ranks_and_error(gpu, eps):
    ttr = _ttr()
    xs = _batch(48, seed=3)
    res = ttr.tt_svd_batched(xs, eps=eps, rmax=16)
    agree = 0
    for x, (cores, ranks, est) in zip(xs, res):
        _, oranks = oracle.tt_svd_eps(x.astype(np.float64), eps, max_ranks=[1] + [16] * (x.ndim - 1) + [1])
        agree += ranks == oranks
        err = oracle.rel_error(x, oracle.tt_full([c.double().cpu().numpy() for c in cores]))
        assert err <= eps * 1.02, (x.shape, ranks, err)
        assert 0.0 <= est <= eps * 1.001
    assert agree >= 46  # sketched steps may round a borderline rank differently


def test_batched_fixed_rank_equals_single_chain(gpu):
    """eps = 0 keeps min(rmax, unfolding size); exact (small-side) steps match the oracle's chain."""
    ttr = _ttr()
    xs = _batch(8, seed=5, dmin=4, dmax=12, rmax=6)
    res = ttr.tt_svd_batched(xs, eps=0.0, rmax=6)
    for x, (cores, ranks, _) in zip(xs, res):
        n = list(x.shape)
        exp = [1]
        left, right = 1, int(np.prod(n))
        for k in range(len(n) - 1):
            left *= n[k]
            right //= n[k]
            exp.append(min(6, left if k == 0 else exp[-1] * n[k], right))
        exp.append(1)
        assert ranks == exp
        ocores, _ = oracle.tt_svd(x.astype(np.float64), exp, method="gram")
        err = oracle.rel_error(x, oracle.tt_full([c.double().cpu().numpy() for c in cores]))
        oerr = oracle.rel_error(x, oracle.tt_full(ocores))
        assert abs(err - oerr) < 1e-3


def test_batched_rejects_bad_arguments(gpu):
    ttr = _ttr()
    from tensor_train_ring_decompositions_hpc_gpu_b200._lib import TTError
    with pytest.raises(TTError):
        ttr.tt_svd_batched([np.ones((4, 4, 4), np.float32)], eps=1e-2, rmax=64)


def test_plan_graph_replay_matches_one_shot_call(gpu):
    """Every autotuner variant (chunk width x work order) and the graph replay give the same
    ranks and cores as the one-shot tt_svd_batched call: the variants change the schedule,
    not the arithmetic of a tensor (each tensor is decomposed by one CTA in a fixed order)."""
    import torch
    ttr = _ttr()
    xs = _batch(40, seed=9)
    ref = ttr.Batch(xs, rmax=16)
    ref.run(eps=1e-2, graph=False)
    b = ttr.Batch(xs, rmax=16)
    b.make_plan(eps=1e-2)
    ms = b.tune(reps=1)
    assert len(ms) == 6 and all(v > 0 for v in ms)
    chunk, largest_first = b.variant()
    assert chunk in (16, 32, 64)
    for _ in range(3):  # first run captures the graph, the others replay it
        b.cores.zero_()
        b.run(eps=1e-2)
        assert list(b.ranks) == list(ref.ranks)
        assert torch.equal(b.cores, ref.cores)
        assert list(b.err) == list(ref.err)
    b.close()


def test_plan_recaptures_for_new_buffers(gpu):
    import torch
    ttr = _ttr()
    xs = _batch(12, seed=10)
    b = ttr.Batch(xs, rmax=16)
    b.run(eps=1e-2)
    first = b.cores.clone()
    b.cores = torch.zeros_like(b.cores)  # a different output buffer: the plan re-captures
    b.run(eps=1e-2)
    assert torch.equal(b.cores, first)
    b.close()
