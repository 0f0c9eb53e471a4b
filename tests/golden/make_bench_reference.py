"""Exact-chain reconstruction errors of the bench.py tensors, computed by the oracle on the CPU.

Rebuilds the bench tensor of a workload (32^6 TT ranks 32, or 32^6 TR bonds 8; seed as in
bench.py) on the CPU: the clean tensor with bench.py's own torch code on the CPU generator, the
noise with the oracle's restatement of the library's Philox generator (seed + 1, stream 7).
Then runs the oracle's exact Gram-eigen chain (the reference's order-6 per-unfolding step,
TT6:510-536, in FP64) and stores the relative reconstruction error and the leading singular
values of every unfolding in bench_reference.json, which bench.py reports next to its own.

    python tests/golden/make_bench_reference.py tt6 [--seed 20261203]

Needs about 50 GB of host memory for the TR workload and a few minutes of CPU time.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def philox_noise(total: int, seed: int, stream: int, chunk_calls: int = 1 << 24) -> np.ndarray:
    """oracle.gaussian_from_philox(total, 1, seed, stream), computed in chunks."""
    out = np.empty(total, dtype=np.float32)
    calls = (total + 3) // 4
    key = (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    for c0 in range(0, calls, chunk_calls):
        c1 = min(calls, c0 + chunk_calls)
        idx = np.arange(c0, c1, dtype=np.uint64)
        ctr = np.zeros((c1 - c0, 4), dtype=np.uint32)
        ctr[:, 0] = idx.astype(np.uint32)
        ctr[:, 1] = np.uint32(stream)
        ctr[:, 2] = (idx >> np.uint64(32)).astype(np.uint32)
        w = oracle.philox4x32_10(ctr, key).astype(np.float64)
        u = (w + 0.5) * (2.0 ** -32)
        r0 = np.sqrt(-2.0 * np.log(u[:, 0]))
        r1 = np.sqrt(-2.0 * np.log(u[:, 2]))
        g = np.empty((c1 - c0, 4))
        g[:, 0] = r0 * np.cos(2 * np.pi * u[:, 1])
        g[:, 1] = r0 * np.sin(2 * np.pi * u[:, 1])
        g[:, 2] = r1 * np.cos(2 * np.pi * u[:, 3])
        g[:, 3] = r1 * np.sin(2 * np.pi * u[:, 3])
        flat = g.ravel()
        e0, e1 = 4 * c0, min(total, 4 * c1)
        out[e0:e1] = flat[: e1 - e0]
    return out


def bench_tensor(name: str, seed: int) -> tuple[np.ndarray, dict]:
    import bench  # noqa: E402  (the repository's bench.py: same generator code)
    wl = dict(bench.WORKLOADS[name])
    x = bench.clean_tensor_torch(wl, seed, "cpu").numpy().astype(np.float32)
    nrm = float(np.linalg.norm(x.astype(np.float64)))
    noise = philox_noise(x.size, seed + 1, 7)
    x += np.float32(wl["noise"] * nrm / np.sqrt(x.size)) * noise
    return x, wl


def chain_error(x: np.ndarray, wl: dict):
    """Exact FP64 Gram-eigen chain; error from ||X - X^||^2 = ||X||^2 - ||X^||^2 (every step is
    an orthogonal projection of the data, so the reconstruction is one too).  For a TR whose
    step-1 rank r0*r1 exceeds n1 this needs the carried rank n1 to be a multiple of r0 (whole
    b-slices of the split are zero, as in the 32^6 TR with r0 = 8); otherwise compare with
    oracle.tr_full instead."""
    shape, ranks = wl["shape"], wl["ranks"]
    xt = x.reshape(shape, order="F")
    if wl["ring"]:
        cores, sig = oracle.tr_svd(xt, ranks, method="gram")
    else:
        cores, sig = oracle.tt_svd(xt, ranks, method="gram")
    nx2 = float(np.sum(x.astype(np.float64) ** 2))
    last = cores[-1]
    nh2 = float(np.sum(np.asarray(last, dtype=np.float64) ** 2))
    err = float(np.sqrt(max(nx2 - nh2, 0.0) / nx2))
    return err, [list(map(float, np.asarray(s)[: min(len(s), 64)])) for s in sig]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["tt6", "tr6", "tt3"])
    ap.add_argument("--seed", type=int, default=20261203)
    args = ap.parse_args()
    t0 = time.time()
    x, wl = bench_tensor(args.workload, args.seed)
    err, sig = chain_error(x, wl)
    path = os.path.join(HERE, "bench_reference.json")
    data = json.load(open(path)) if os.path.exists(path) else {}
    data[args.workload] = {"seed": args.seed, "rel_err_exact": err, "sigma": sig,
                           "method": "oracle exact Gram-eigen chain, FP64", "cpu_seconds": time.time() - t0}
    with open(path, "w") as f:
        json.dump(data, f, indent=1)
    print(args.workload, "exact-chain rel err", err, f"({time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
