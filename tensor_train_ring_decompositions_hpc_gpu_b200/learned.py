"""Training data, training run and weights of the learned EDrSVD parameter predictor.

The predictor (kernels in ``csrc/mlp.cu``) maps 8 Gaussian-probe features of an unfolding
(``tt_probe_features``) to its truncation rank, oversampling and power-iteration count.  This
module builds its training set and trains it with the library's own GPU kernels:

* Unfoldings: spectra of a low-rank tensor with noise, sigma_i = i^-alpha for i <= R (the bond
  dimension, R ~ U{8..112}, alpha ~ U[0.5, 2]) and a flat noise floor holding a share eta^2 of
  the energy beyond R (eta log-uniform in [1e-6, tol / 4]), k = min(m, n) log-uniform in
  [129, 2048] (sizes where a TT step of an order-6 tensor with modes 24..40 takes the randomized
  path), and a step tolerance tol log-uniform in [2e-4, 3e-3] (the per-unfolding share
  eps / sqrt(d - 1) of eps = 1e-3 for orders 2..6, with margin).  The eps-rank is then at most
  R + a few, within the 128-column sketch limit, so every label is a reachable target.
* Features: ``tt_probe_features`` on the k x k matrix diag(sigma).  For A = U diag(sigma) V^T
  with orthonormal U, V and a Gaussian probe Omega, V^T Omega is Gaussian again, so the probe
  statistics (and every EDrSVD quantity) of A and of diag(sigma) have the same distribution.
* Labels (the plain method in FP64): the rank r* of the exact truncated SVD at tolerance tol
  (smallest r with sum_{i>r} sigma_i^2 <= tol^2 sum sigma_i^2), and the cheapest (power
  iterations p, oversampling s) for which the EDrSVD with r* + s columns, its passes over A
  perturbed by the tensor cores' TF32 operand rounding (the engine the learned form runs on),
  leaves at most half of tol^2 of the energy outside its subspace in every trial (the half
  leaves room for the noise of the probe-based a-posteriori estimate that judges a learned
  attempt): fewer passes over A first (2 + 2p), then the narrower sketch.
* Training: ``tt_mlp_train`` (Adam, one persistent launch), on 90 % of the samples; the rest
  measure the validation loss.

``python -m tensor_train_ring_decompositions_hpc_gpu_b200.learned labels --out FILE.npz`` computes
the specifications and labels on the CPU; ``... learned train --data FILE.npz --out FILE.npy``
adds the probe features and trains on a GPU (without --data it labels first);
``... learned evaluate`` compares the shipped predictor with the plain adaptive method.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _lib

RANK_CAP = 120            # largest rank the randomized step can return (sketch width <= 128)
OVERSAMPLE = (4, 8, 16, 32)
POWER = (0, 1, 2)
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "predictor_weights.npy")


def sample_specs(count, seed, kmin=129, kmax=2048, amin=0.5, amax=2.0, tmin=2e-4, tmax=3e-3, rmin=8, rmax=112):
    """(k, alpha, tol, R, eta) of `count` training unfoldings."""
    rng = np.random.default_rng(seed)
    k = np.exp(rng.uniform(np.log(kmin), np.log(kmax + 1), count)).astype(np.int64)
    alpha = rng.uniform(amin, amax, count)
    tol = np.exp(rng.uniform(np.log(tmin), np.log(tmax), count))
    bond = np.minimum(rng.integers(rmin, rmax + 1, count), k - 1)
    eta = np.exp(rng.uniform(np.log(1e-6), np.log(tol / 4.0)))
    return k, alpha, tol, bond, eta


def spectrum(k, alpha, bond=None, eta=0.0):
    """sigma_i = i^-alpha for i <= bond, then a flat floor carrying a share eta^2 of the energy."""
    k = int(k)
    bond = k if bond is None else int(bond)
    sig = np.zeros(k, dtype=np.float64)
    sig[:bond] = np.arange(1, bond + 1, dtype=np.float64) ** (-float(alpha))
    if bond < k and eta > 0.0:
        e = float(np.sum(sig[:bond] ** 2))
        sig[bond:] = np.sqrt(eta * eta * e / (1.0 - eta * eta) / (k - bond))
    return sig


def exact_rank(sig, tol, cap=RANK_CAP):
    """Smallest r with sum_{i>r} sigma_i^2 <= tol^2 ||sigma||^2 (the exact FP64 truncated SVD)."""
    e = sig * sig
    tail = np.concatenate([np.cumsum(e[::-1])[::-1], [0.0]])  # tail[r] = sum_{i>=r} e_i (0-based)
    ok = np.nonzero(tail <= tol * tol * e.sum())[0]
    r = int(ok[0]) if ok.size else int(sig.size)
    return max(1, min(r, cap))


def _orth(y):
    q, _ = np.linalg.qr(y)
    return q


# Relative RMS of the TF32 rounding of an FP32 operand (10 stored mantissa bits, round to
# nearest): the learned form's sketch and power passes run on the tensor cores, and this white
# noise, about as strong per direction as a 1e-4 noise floor, perturbs the captured range.
TF32_NOISE = 2.5e-4


def edrsvd_outside(sig, ks, p, rng, op_noise=TF32_NOISE):
    """Energy share outside the EDrSVD subspace of A = diag(sig) (ks columns, p power
    iterations), every pass over A seeing A plus fresh white noise of relative RMS op_noise per
    element of a dense A of the same spectrum (the tensor cores' operand rounding)."""
    k = sig.size
    e = sig * sig
    g_sd = op_noise * np.sqrt(e.sum()) / k  # per-entry sd: ||G||_F = op_noise ||A||_F

    def mul(x):  # (A + G) x with a fresh G
        out = sig[:, None] * x
        if g_sd > 0.0:
            out += g_sd * (rng.standard_normal((k, k)) @ x)
        return out
    q = _orth(mul(rng.standard_normal((k, ks))))
    for _ in range(p):
        z = _orth(mul(q))               # A^T Q (A = diag(sig) is symmetric)
        q = _orth(mul(z))               # A Z
    captured = float(np.sum(e[:, None] * q * q))
    return max(e.sum() - captured, 0.0) / e.sum()


def label(k, alpha, tol, seed, bond=None, eta=0.0, trials=2):
    """(r*, s*, p*, feasible) of one unfolding: the eps-rank and the cheapest (p, s) whose FP64
    EDrSVD leaves at most tol^2 / 2 outside its subspace in every trial.  A rank above RANK_CAP
    (not reached by this distribution) is labelled with the widest sketch and p = 1."""
    sig = spectrum(k, alpha, bond, eta)
    r = exact_rank(sig, tol, cap=int(k))
    if r > RANK_CAP:
        return RANK_CAP, 8, 1, False
    rng = np.random.default_rng(seed)
    for p in POWER:
        for s in OVERSAMPLE:
            ks = min(r + s, _lib.TT_MAX_SMALL, int(k))
            if all(edrsvd_outside(sig, ks, p, rng) <= 0.5 * tol * tol for _ in range(trials)):
                return r, s, p, True
    return r, OVERSAMPLE[-1], POWER[-1], False


def _label_chunk(args):
    k, alpha, tol, bond, eta, seeds, one_thread = args
    rows = list(zip(k, alpha, tol, bond, eta, seeds))

    def run():
        return [label(int(a), float(b), float(c), int(f), int(d), float(e)) for a, b, c, d, e, f in rows]
    if one_thread:  # one BLAS thread per pool worker: the pool already fills the cores
        from threadpoolctl import threadpool_limits
        with threadpool_limits(1):
            return run()
    return run()


def labels(k, alpha, tol, bond, eta, seed, workers=None):
    """Labels of all samples, over a spawn process pool (started before any GPU call)."""
    seeds = np.random.default_rng(seed + 1).integers(1 << 31, size=k.size)
    workers = workers or max(1, min(32, len(os.sched_getaffinity(0))))
    chunks = np.array_split(np.arange(k.size), workers * 4)
    jobs = [(k[c], alpha[c], tol[c], bond[c], eta[c], seeds[c], workers > 1) for c in chunks]
    if workers == 1:
        res = [_label_chunk(j) for j in jobs]
    else:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            res = pool.map(_label_chunk, jobs)
    out = np.array([x for part in res for x in part], dtype=np.float64)
    return out[:, 0], out[:, 1], out[:, 2], out[:, 3].astype(bool)


def targets(r, s, p):
    """Network targets: log2 r / 10, log2 s / 5, p / 2 (decoded by the library as
    round(2^(10 y0)), round(2^(5 y1)), round(2 y2))."""
    return np.stack([np.log2(r) / 10.0, np.log2(s) / 5.0, p / 2.0], axis=1).astype(np.float32)


def features(k, alpha, tol, seed, bond, eta, device=None, log=None):
    """Probe features of diag(sigma) for every sample, computed by tt_probe_features."""
    import torch
    from . import probe_features
    dev = device or torch.device("cuda")
    out = torch.empty((k.size, _lib.TT_MLP_INPUTS), dtype=torch.float32, device=dev)
    t0 = time.time()
    for i in range(k.size):
        sig = spectrum(k[i], alpha[i], bond[i], eta[i])
        a = torch.diag(torch.from_numpy(sig).float().to(dev))  # symmetric: its column-major view is itself
        e = float(np.sum(sig * sig))
        out[i] = probe_features(a, energy=e, tol=float(tol[i]), seed=int(seed) + i, stream_id=0)
        if log and (i + 1) % 5000 == 0:
            log(f"features {i + 1}/{k.size}: {time.time() - t0:.1f} s")
    return out.cpu().numpy()


def init_params(seed):
    """He-uniform weights, zero biases, packed W1 b1 W2 b2 W3 b3."""
    rng = np.random.default_rng(seed)
    parts = []
    for rows, cols in ((64, 8), (64, 64), (3, 64)):
        lim = np.sqrt(6.0 / cols)
        parts += [rng.uniform(-lim, lim, rows * cols), np.zeros(rows)]
    return np.concatenate(parts).astype(np.float32)


def train(x, t, steps=8000, batch=256, lr=1e-3, seed=7, device=None, log=None):
    """Train on the GPU with tt_mlp_train; returns (params as NumPy, loss trace)."""
    import torch
    from . import mlp_train
    dev = device or torch.device("cuda")
    p = torch.from_numpy(init_params(seed)).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    xt = torch.from_numpy(x).to(dev)
    tt = torch.from_numpy(t).to(dev)
    traces, done = [], 0
    # two phases: lr, then lr / 4 for the last quarter
    for n_steps, rate in ((steps - steps // 4, lr), (steps // 4, lr / 4)):
        traces.append(mlp_train(p, m, v, xt, tt, n_steps, batch=batch, lr=rate, step0=done, seed=seed).cpu().numpy())
        done += n_steps
        if log:
            log(f"step {done}: minibatch loss {float(traces[-1][-20:].mean()):.5f}")
    return p.cpu().numpy(), np.concatenate(traces)


def decode(y, ks_cap=_lib.TT_MAX_SMALL):
    """(rank, oversampling, power iterations, sketch width) the library derives from outputs y."""
    y = np.asarray(y, dtype=np.float64)
    r = np.maximum(1.0, np.rint(np.exp2(np.minimum(10.0 * y[..., 0], 10.0))))
    s = np.rint(np.exp2(np.clip(5.0 * y[..., 1], 1.0, 5.0)))
    p = np.rint(np.clip(2.0 * y[..., 2], 0.0, 3.0))
    ks = np.clip(r + s, 1, ks_cap)
    ks = np.where(10 * ks >= 9 * ks_cap, ks_cap, ks)  # the library snaps widths within 10 % to the limit
    return r.astype(int), s.astype(int), p.astype(int), ks.astype(int)


def save_params(path, params):
    np.save(path, np.asarray(params, dtype=np.float32).ravel())


def load_params(path=WEIGHTS):
    p = np.load(path).astype(np.float32).ravel()
    if p.size != _lib.TT_MLP_PARAMS:
        raise ValueError(f"{path}: {p.size} parameters, expected {_lib.TT_MLP_PARAMS}")
    return p


def label_dataset(count, seed, workers=None, log=None):
    """Specifications and labels (CPU only) of `count` training unfoldings."""
    log = log or (lambda msg: print(msg, flush=True))
    t0 = time.time()
    k, alpha, tol, bond, eta = sample_specs(count, seed)
    r, s, p, feas = labels(k, alpha, tol, bond, eta, seed, workers)
    log(f"labels of {count} unfoldings: {time.time() - t0:.1f} s, feasible {feas.mean():.3f}")
    return dict(k=k, alpha=alpha, tol=tol, bond=bond, eta=eta, r=r, s=s, p=p, feasible=feas, seed=seed)


def add_features(data, log=None):
    """The probe features (GPU) and network targets of a labelled set."""
    log = log or (lambda msg: print(msg, flush=True))
    t0 = time.time()
    data = dict(data)
    data["x"] = features(data["k"], data["alpha"], data["tol"], int(data["seed"]), data["bond"], data["eta"],
                         log=log)
    data["t"] = targets(data["r"], data["s"], data["p"])
    log(f"features: {time.time() - t0:.1f} s")
    return data


def evaluate(weights=WEIGHTS, count=24, n=32768, tol=1e-3, seed=5, reps=3, log=None):
    """Learned against plain adaptive EDrSVD on `count` held-out unfoldings U diag(sigma) V^T
    with the training distribution's spectra (m ~ U{200..1024}, bond R ~ U{8..112}, alpha ~
    U[0.5, 2], noise floor eta ~ logU[1e-6, tol / 4]; orthonormal U, V drawn on the GPU): passes
    over A, device time (median of `reps` after a warm-up), achieved error and its estimate."""
    import torch
    from . import TT_FLAG_ADAPTIVE_KS, TT_FLAG_LEARNED, set_predictor, tt_svd
    dev = torch.device("cuda", 0)
    set_predictor(load_params(weights))
    rng = np.random.default_rng(seed)
    rows = []
    try:
        for i in range(count):
            m = int(rng.integers(200, 1025))
            alpha = float(rng.uniform(0.5, 2.0))
            bond = int(rng.integers(8, 113))
            eta = float(np.exp(rng.uniform(np.log(1e-6), np.log(tol / 4.0))))
            g = torch.Generator(device=dev).manual_seed(i)
            u, _ = torch.linalg.qr(torch.randn(m, m, generator=g, device=dev))
            v, _ = torch.linalg.qr(torch.randn(n, m, generator=g, device=dev))
            sig = torch.from_numpy(spectrum(m, alpha, bond, eta)).float().to(dev)
            a = (u * sig) @ v.T
            out = {"m": m, "n": n, "alpha": alpha, "bond": bond, "eta": eta}
            for name, flags in (("plain", TT_FLAG_ADAPTIVE_KS), ("learned", TT_FLAG_LEARNED)):
                tt_svd(a, [1, 120, 1], eps=tol, power_iters=1, flags=flags)
                ms = []
                for _ in range(reps):
                    res = tt_svd(a, [1, 120, 1], eps=tol, power_iters=1, flags=flags)
                    ms.append(res.ms)
                uu = res.cores[0].reshape(m, -1).double()
                ww = res.cores[1].reshape(res.cores[1].shape[0], -1).double()
                err = float(torch.linalg.matrix_norm(a.double() - uu @ ww) / torch.linalg.matrix_norm(a.double()))
                out[name] = dict(ms=float(np.median(ms)), passes=res.passes, ks=res.step_ks[0], p=res.step_power[0],
                                 attempts=res.step_attempts[0], fallbacks=res.fallbacks, rank=res.ranks[1],
                                 est=res.est_rel_err, err=err, eps_unmet=res.eps_unmet)
            rows.append(out)
            if log:
                log(json.dumps(out))
    finally:
        set_predictor(None)
    summ = {"unfoldings": count, "tol": tol,
            "passes_plain": int(sum(r["plain"]["passes"] for r in rows)),
            "passes_learned": int(sum(r["learned"]["passes"] for r in rows)),
            "ms_plain": float(sum(r["plain"]["ms"] for r in rows)),
            "ms_learned": float(sum(r["learned"]["ms"] for r in rows)),
            "fallbacks": int(sum(r["learned"]["fallbacks"] for r in rows)),
            "max_err_ratio_learned_over_plain": float(max(r["learned"]["err"] / r["plain"]["err"] for r in rows))}
    return summ, rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    lb = sub.add_parser("labels")
    lb.add_argument("--count", type=int, default=20000)
    lb.add_argument("--seed", type=int, default=20261203)
    lb.add_argument("--workers", type=int, default=None)
    lb.add_argument("--out", required=True, help="labelled set (.npz)")
    tr = sub.add_parser("train")
    tr.add_argument("--data", default=None, help="labelled set from `labels` (default: label here first)")
    tr.add_argument("--count", type=int, default=20000)
    tr.add_argument("--steps", type=int, default=8000)
    tr.add_argument("--batch", type=int, default=256)
    tr.add_argument("--lr", type=float, default=1e-3)
    tr.add_argument("--seed", type=int, default=20261203)
    tr.add_argument("--workers", type=int, default=None)
    tr.add_argument("--out", required=True)
    tr.add_argument("--report", default=None, help="JSON summary of the run")
    ev = sub.add_parser("evaluate")
    ev.add_argument("--weights", default=WEIGHTS)
    ev.add_argument("--count", type=int, default=24)
    ev.add_argument("--tol", type=float, default=1e-3)
    args = ap.parse_args(argv)
    if args.cmd == "evaluate":
        summ, _ = evaluate(args.weights, args.count, tol=args.tol, log=lambda msg: print(msg, flush=True))
        print(json.dumps({"summary": summ}))
        return 0
    if args.cmd == "labels":
        data = label_dataset(args.count, args.seed, args.workers)
        np.savez_compressed(args.out, **data)
        return 0
    if args.data:
        data = {key: val for key, val in np.load(args.data).items()}
    else:
        data = label_dataset(args.count, args.seed, args.workers)  # the pool runs before the first GPU call
    data = add_features(data)
    args.count = int(data["k"].size)
    n = args.count
    ntr = int(0.9 * n)
    t0 = time.time()
    params, trace = train(data["x"][:ntr], data["t"][:ntr], steps=args.steps, batch=args.batch, lr=args.lr,
                          seed=args.seed, log=lambda msg: print(msg, flush=True))
    train_s = time.time() - t0
    import torch
    from . import mlp_forward
    y = mlp_forward(torch.from_numpy(params).cuda(), torch.from_numpy(data["x"][ntr:]).cuda()).cpu().numpy()
    val = float(np.mean(np.sum((y - data["t"][ntr:]) ** 2, axis=1)))
    r, s, p, ks = decode(y)
    rt = data["r"][ntr:]
    save_params(args.out, params)
    rep = {"samples": n, "train": ntr, "steps": args.steps, "batch": args.batch, "train_seconds": train_s,
           "final_minibatch_loss": float(trace[-50:].mean()), "validation_loss": val,
           "validation_rank_within_10pct": float(np.mean(np.abs(r - rt) <= 0.1 * rt + 1)),
           "validation_power_exact": float(np.mean(p == data["p"][ntr:])),
           "feasible_share": float(data["feasible"].mean())}
    print(json.dumps(rep))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
