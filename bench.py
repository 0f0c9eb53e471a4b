"""Benchmark of the TT-SVD / TR-SVD hot path on B200.

Headline workload (one "step"): the order-6 TT-SVD of a 32^6 FP32 tensor (4.29 GB) built from
random TT cores with ranks (1,32,32,32,32,32,1), N(0,1) entries and 1e-4-relative Gaussian
noise, decomposed back to those ranks with the randomized EDrSVD chain (oversampling 8, no
power iteration, TF32 tensor cores for the bulk passes).  Synthetic data; the tensor is 34x the
126 MB L2, so no L2 flush is needed between steps.

The same JSON line carries, under ``workloads``, the other configurations measured in the same
run on the same GPU: ``tt3`` (plain third-order TT-SVD, 256^3 FP32, ranks 16, s = 8, p = 1, FP32
CUDA-core GEMMs), ``tr6`` (order-6 TR-SVD, 32^6, bond ranks 8), ``batch4`` (4096 order-4 tensors
in one persistent launch) and ``c5`` (learned vs plain adaptive EDrSVD on order-6 tensors with
power-law unfolding spectra).  ``--workload`` runs one of them alone as the headline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  ``value`` is whole-job TFLOP/s: the algorithmic FLOPs of the
executed chain (the library's plan restated below; checked against the library's own count)
times the number of ranks, divided by the slowest rank's device time per step.  Multi-GPU runs
are independent replicas (each rank decomposes its own tensor; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "order-6 TT/TR-SVD ms & TFLOP/s at rel err ≤1e-3; learned+BF16 vs plain FP32"

WORKLOADS = {
    "tt6": dict(shape=[32] * 6, ranks=[1, 32, 32, 32, 32, 32, 1], ring=False, noise=1e-4, gemm="auto",
                desc="order-6 TT-SVD, 32^6 FP32, TT ranks (1,32,32,32,32,32,1), 1e-4 noise"),
    # The TR's unfoldings have flat spectra around the rank-8 cut (sigma_8 / sigma_9 = 1.013 in
    # unfolding 2) and rank r0 r_k = 64 above the noise: a sketch of 80 columns with one power
    # iteration (and the exact, refined step of the 128-row unfolding 2) meets the leading
    # singular values of the exact chain within 1e-4; narrower or power-free sketches do not.
    "tr6": dict(shape=[32] * 6, ranks=[8, 8, 8, 8, 8, 8, 8], ring=True, noise=1e-4, oversample=72, power_iters=1,
                gemm="auto", desc="order-6 TR-SVD, 32^6 FP32, bond ranks 8 (first split 64), 1e-4 noise"),
    "tt3": dict(shape=[256] * 3, ranks=[1, 16, 16, 1], ring=False, noise=1e-3, oversample=8, power_iters=1,
                gemm="fp32", flush_l2=True,
                desc="plain third-order TT-SVD, 256^3 FP32, ranks (1,16,16,1), 1e-3 noise, s = 8, p = 1, "
                     "FP32 CUDA-core GEMMs"),
}
MAX_SMALL = 128  # TT_MAX_SMALL: widest exact step / sketch


# ---------------------------------------------------------------------------------------
# algorithmic work of the executed chain: the library's plan (make_plan in csrc/driver.cu)
# restated, so that the CPU arm can use the same FLOP numerator; checked against the
# library's own count (tt_stats.flops) in every run
# ---------------------------------------------------------------------------------------
def plan_steps(shape, ranks, ring, s=8):
    """Per unfolding: rows m, columns, path (exact rows / exact columns / randomized), sketch
    width, rows written for the next unfolding (row compaction of zero-padded ranks), fold."""
    d = len(shape)
    size = int(np.prod(shape))
    rows_prev = 1
    steps = []
    for k in range(d - 1):
        first_ring = ring and k == 0
        m = shape[0] if first_ring else rows_prev * shape[k]
        cols = size // m
        rq = ranks[0] * ranks[1] if first_ring else ranks[k + 1]
        mn = min(m, cols)
        re = min(rq, mn)
        small_exact = mn <= 64 or (mn <= MAX_SMALL and 2 * (re + s) >= mn)
        if small_exact:
            path, ks = ("rows" if m <= cols else "cols"), mn
        else:
            path, ks = "rand", min(re + s, mn, MAX_SMALL)
        fold = (not (ring and k == 0)) and path == "rows" and rq == m and re == m and rows_prev == ranks[k]
        if first_ring:
            r1_out = -(-re // ranks[0])
            n_out = ranks[0] * r1_out
        else:
            r1_out = 0
            n_out = rq if fold else re
        steps.append(dict(m=m, cols=cols, rq=rq, re=re, ks=ks, path=path, fold=fold, n_out=n_out))
        if not fold:
            size = n_out * cols
        rows_prev = r1_out if first_ring else n_out
    return steps


def chain_flops(shape, ranks, ring, s=8, p=0, gemm="auto"):
    """FLOPs the library counts for a fixed-rank chain (same terms as its pass accounting).
    An exact step over more than 32 rows that truncates (not the TR bond split) and whose Gram
    runs on the tensor cores (gemm "tc", or "auto" on an unfolding of at least 2^24 elements)
    replaces the projection by an exact Rayleigh-Ritz refinement on b = r + 16 eigenvectors:
    Z = A^T U0, the Gram of Z and the next data E_r^T Z^T."""
    fl = 0.0
    for k, st in enumerate(plan_steps(shape, ranks, ring, s)):
        m, cols, ks, nout = st["m"], st["cols"], st["ks"], st["n_out"]
        if st["path"] == "rows":
            fl += 2.0 * m * m * cols
            tc = gemm == "tc" or (gemm == "auto" and m * cols >= 1 << 24)
            refine = tc and m > 32 and st["re"] < m and not (ring and k == 0) and not st["fold"]
            if refine:
                b = min(m, st["re"] + 16)
                fl += 2.0 * m * cols * b + 2.0 * cols * b * b + 2.0 * b * cols * nout
            elif not st["fold"]:
                fl += 2.0 * m * cols * nout
        elif st["path"] == "cols":
            fl += 2.0 * m * cols * cols + 2.0 * m * cols * st["rq"]
        else:
            fl += 2.0 * m * cols * ks * (2 + 2 * p)  # sketch, p x (Z = A^T Q, Y = A Z), B = Q^T A
            fl += p * 4.0 * cols * ks * ks           # orthonormalisation of each power basis
            fl += 2.0 * cols * ks * ks               # Gram of B
            fl += 2.0 * ks * cols * nout             # next data = E_r^T B
    return fl


# ---------------------------------------------------------------------------------------
# synthetic inputs
# ---------------------------------------------------------------------------------------
def make_tensor_torch(wl, seed, device):
    """Column-major flat FP32 tensor on the device (torch is used for generation only)."""
    import torch
    x = clean_tensor_torch(wl, seed, device)
    nrm = torch.linalg.vector_norm(x.double()).item()
    # Noise from the library's counter-based Philox generator (seed + 1, stream 7), so the
    # same tensor can be rebuilt on the CPU (tests/golden/make_bench_reference.py).
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    noise = ttr.gaussian(x.numel(), 1, seed=seed + 1, stream_id=7, device=x.device).reshape(-1)
    x.add_(noise, alpha=wl["noise"] * nrm / np.sqrt(x.numel()))
    del noise
    return x.contiguous()


def clean_tensor_torch(wl, seed, device):
    """The noise-free TT/TR tensor (column-major flat FP32) from seeded N(0,1) cores."""
    import torch
    shape, ranks, ring = wl["shape"], wl["ranks"], wl["ring"]
    d = len(shape)
    g = torch.Generator(device="cpu").manual_seed(seed)
    if not ring:
        # The column-major matrix M_k = (r_{k-1} n_k) x rest is held as its row-major transpose
        # T_k.  T_k = T_{k+1}' @ G_k^T, where T_{k+1}' is T_{k+1} re-read as (n_k+1 rest) x r_k
        # (the free column-major reshape of the TT chain).
        mt = torch.randn(shape[-1], ranks[d - 1], generator=g).to(device)
        for k in range(d - 2, -1, -1):
            gt = torch.randn(ranks[k + 1], ranks[k] * shape[k], generator=g).to(device)
            mt = (mt @ gt).reshape(-1, ranks[k])
        x = mt.reshape(-1)
    else:
        x = _tr_full_torch(shape, ranks[0], g, device)
    return x


def _tr_full_torch(shape, bond, g, device):
    import torch
    d = len(shape)
    cores = [torch.randn(bond, shape[k], bond, generator=g).to(device) for k in range(d)]
    # merge cores 2..d: M (r1, N, r0) column-major, built as a torch tensor with logical dims
    m = cores[1]  # (b, i2, c)
    for k in range(2, d):
        m = torch.einsum("bjc,cid->bjid", m, cores[k])
        b, j, i, dd = m.shape
        m = m.permute(0, 2, 1, 3).reshape(b, i * j, dd)  # merged index j + (size j) * i
    # X[i1, J] = sum_{a,b} G1[a,i1,b] M[b,J,a], J = (i2 fastest ... id slowest)
    x = torch.einsum("aib,bja->ji", cores[0], m)  # (N, n1) row-major = column-major (n1 x N)
    return x.reshape(-1).contiguous()


# ---------------------------------------------------------------------------------------
# CPU baseline: the reference's own chain restated in NumPy FP32, full size
# ---------------------------------------------------------------------------------------
def _gram_eig_cpu(a, r):
    """One step of the reference's order-6 chain (longMatrixSVD_Eign_once_device, TT6:510-536):
    W = A A^T, eigenvectors in descending order, the top r of them (G), next = G^T A written
    column-major (r x cols)."""
    w = a @ a.T
    lam, v = np.linalg.eigh(w.astype(np.float64))
    k = min(r, a.shape[0])
    g = np.ascontiguousarray(v[:, ::-1][:, :k].astype(np.float32))
    return (a.T @ g).T, k  # (cols x k) C-order = (k x cols) column-major, no transposing copy


def _edrsvd_cpu(a, r, s, p, rng):
    """Plain EDrSVD (basicRandSVD, EDR:175-326): Gaussian Omega, Y = A Omega, QR, p power
    iterations, B = Q^T A, SVD of B; returns S V^T (r x cols, column-major)."""
    m, n = a.shape
    ks = min(r + s, m, n)
    om = rng.standard_normal((n, ks), dtype=np.float32)
    q, _ = np.linalg.qr(a @ om)
    for _ in range(p):
        z, _ = np.linalg.qr(a.T @ q)
        q, _ = np.linalg.qr(a @ z)
    b = (a.T @ q).T
    _, sv, vt = np.linalg.svd(b, full_matrices=False)
    k = min(r, ks)
    return np.asfortranarray(sv[:k, None] * vt[:k]), k


def cpu_chain(xh, wl, s=8, p=1):
    """Seconds for one full-size decomposition on the host cores: the order-6 Gram-eigen chain of
    TT6:799-958 / TR6:827-1004 (with the 231 permute of TR6:49-58 after the ring's first step),
    or, for the third-order workload, the plain EDrSVD chain of EDR:329-586."""
    shape, ranks, ring = wl["shape"], wl["ranks"], wl["ring"]
    d = len(shape)
    rng = np.random.default_rng(0)
    t0 = time.perf_counter()
    flat = xh
    rows_prev = 1
    for k in range(d - 1):
        first_ring = ring and k == 0
        m = shape[0] if first_ring else rows_prev * shape[k]
        a = flat.reshape(m, flat.size // m, order="F")
        rq = ranks[0] * ranks[1] if first_ring else ranks[k + 1]
        if d == 3 and not ring:
            nxt, re = _edrsvd_cpu(a, rq, s, p, rng)
        else:
            nxt, re = _gram_eig_cpu(a, rq)
        if first_ring:
            r0 = ranks[0]
            r1e = -(-re // r0)
            if r0 * r1e > re:
                nxt = np.vstack([nxt, np.zeros((r0 * r1e - re, nxt.shape[1]), dtype=np.float32)])
            # (r0, r1, N) -> (r1, N, r0), column-major
            t = np.asfortranarray(nxt).reshape(r0, r1e, -1, order="F").transpose(1, 2, 0)
            flat = t.ravel(order="F")
            rows_prev = r1e
        else:
            flat = nxt.ravel(order="F")
            rows_prev = re
    return time.perf_counter() - t0


def host_tensor(wl, seed):
    """The workload's tensor on the host (clean part with the bench's own generator on the CPU,
    noise from NumPy): same distribution as the device tensor, built without the GPU."""
    x = clean_tensor_torch(wl, seed, "cpu").numpy().astype(np.float32, copy=False)
    nrm = float(np.linalg.norm(x.astype(np.float64)))
    rng = np.random.default_rng(seed + 1)
    x += np.float32(wl["noise"] * nrm / np.sqrt(x.size)) * rng.standard_normal(x.size, dtype=np.float32)
    return x


def cpu_baseline(xh, wl, args, steps, budget_s=90.0):
    """Time `steps` full-size decompositions (after one untimed warm-up) on the host cores;
    stops early when the budget runs out (the number timed is reported)."""
    s, p = wl_sp(wl, args)
    cpu_chain(xh, wl, s, p)
    ts = []
    t_start = time.perf_counter()
    for _ in range(steps):
        ts.append(cpu_chain(xh, wl, s, p))
        if time.perf_counter() - t_start > budget_s:
            break
    return float(np.mean(ts)), len(ts)


def wl_sp(wl, args):
    s = args.oversample if args.oversample is not None else wl.get("oversample", 8)
    p = args.power_iters if args.power_iters is not None else wl.get("power_iters", 0)
    return s, p


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        info = threadpool_info()
        return max([i.get("num_threads", 1) for i in info if i.get("user_api") == "blas"] or [1])
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def exact_chain_parity(key, seed, wl, rel_err, st):
    """Compare with the oracle's exact FP64 chain on the same tensor (tests/golden/
    bench_reference.json, made by tests/golden/make_bench_reference.py): reconstruction error
    gap and, per unfolding, the relative deviation of the singular values up to its target rank
    (largest deviation, and how many leading ones are within 1e-4)."""
    path = os.path.join(ROOT, "tests", "golden", "bench_reference.json")
    try:
        ref = json.load(open(path)).get(key)
    except Exception:
        ref = None
    if not ref or ref.get("seed") != seed or wl.get("override"):
        return None
    ranks, ring = wl["ranks"], wl["ring"]
    per_step = []
    for k in range(min(len(ref["sigma"]), int(st.nsteps))):
        rk = ranks[0] * ranks[1] if (ring and k == 0) else ranks[k + 1]
        mine = np.array(st.sigma[k][: st.nsigma[k]], dtype=np.float64)
        theirs = np.array(ref["sigma"][k], dtype=np.float64)
        cnt = min(rk, mine.size, theirs.size, int(np.sum(theirs > 1e-6 * theirs[0])))
        rel = np.abs(mine[:cnt] - theirs[:cnt]) / theirs[:cnt] if cnt > 0 else np.zeros(0)
        lead = int(np.argmax(rel > 1e-4)) if np.any(rel > 1e-4) else int(cnt)
        per_step.append({"compared": int(cnt), "max_rel_dev": float(np.max(rel)) if cnt else None,
                         "leading_within_1e-4": lead})
    devs = [p["max_rel_dev"] for p in per_step if p["max_rel_dev"] is not None]
    return {"rel_err_exact_chain": ref["rel_err_exact"], "rel_err_gap": abs(rel_err - ref["rel_err_exact"]),
            "sigma_max_rel_dev": max(devs) if devs else None, "sigma_per_unfolding": per_step,
            "reference": "oracle exact Gram-eigen chain (FP64) on this tensor"}


def committed_traffic(workload, key):
    """DRAM bytes (read + write) per launch of one pass, from a committed ncu capture."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            v = json.load(f).get(workload, {}).get(key)
        return None if v is None else float(v["bytes"])
    except Exception:
        return None


# ---------------------------------------------------------------------------------------
# ---------------------------------------------------------------------------------------
# batched small tensors: 4096 order-4 TT tensors, modes U{8..32}, ranks U{2..16}, 1e-3 noise
# ---------------------------------------------------------------------------------------
BATCH = dict(count=4096, order=4, nmin=8, nmax=32, rmin=2, rmax=16, noise=1e-3, eps=1e-2)


def batch_tensors_torch(seed, device, count=None):
    """Seeded order-4 TT tensors (N(0,1) cores, relative noise) built on the device."""
    import torch
    cfg = BATCH
    count = count or cfg["count"]
    rng = np.random.default_rng(seed)
    g = torch.Generator(device="cpu").manual_seed(seed)
    out = []
    for _ in range(count):
        n = [int(v) for v in rng.integers(cfg["nmin"], cfg["nmax"] + 1, size=cfg["order"])]
        r = [1] + [int(v) for v in rng.integers(cfg["rmin"], cfg["rmax"] + 1, size=cfg["order"] - 1)] + [1]
        cores = [torch.randn(r[k], n[k], r[k + 1], generator=g).to(device) for k in range(cfg["order"])]
        x = cores[0].reshape(n[0], r[1])                      # (i1, a1)
        for k in range(1, cfg["order"]):
            x = torch.einsum("ia,ajb->ijb", x, cores[k]).reshape(-1, r[k + 1])
        xt = x.reshape(*n)  # row-major over (i1, ..., id): the logical tensor
        xt = xt + cfg["noise"] * torch.linalg.vector_norm(xt) / np.sqrt(xt.numel()) * torch.randn(
            xt.shape, generator=g).to(device)
        out.append(xt)
    return out


def measure_batch(args, dev, steps=None, warmup=None):
    """batch4: tensors/s of one graph-replayed persistent launch over the whole batch, the
    autotuned variant, parity on a sample against the oracle's delta-truncation, roofline of
    the launch (the algorithmic bytes: every tensor read once plus its cores written)."""
    import torch
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    steps = steps or min(args.steps, 10)
    warmup = max(warmup or args.warmup, 3)
    xs = batch_tensors_torch(args.seed, dev, count=getattr(args, "batch_count", None))
    b = ttr.Batch(xs, rmax=BATCH["rmax"], device=dev)
    elems = float(b.flat.numel())
    b.make_plan(eps=BATCH["eps"])
    tune_ms = b.tune(reps=2)  # autotuner: sketch chunk width x work order, fastest kept
    chunk, largest_first = b.variant()
    for _ in range(warmup):
        b.run(eps=BATCH["eps"])  # first run captures the CUDA graph
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(dev.index or 0)
    clk.start()
    e0.record()
    for _ in range(steps):
        b.run(eps=BATCH["eps"])
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / steps
    res = b.results()
    ranks = [r for _, r, _ in res]
    errs = np.array([e for _, _, e in res])
    core_elems = float(sum(sum(c.numel() for c in cs) for cs, _, _ in res))
    alg_bytes = 4.0 * (elems + core_elems)
    peak, peak_src = peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    out = {
        "metric": f"batched TT-SVD of {len(xs)} order-4 tensors (eps 1e-2)", "value": len(xs) / (ms * 1e-3),
        "unit": "tensors/s", "ms": ms, "steps": steps, "warmup": warmup,
        "config": {"workload": "batch4: 4096 order-4 TT tensors, modes U{8..32}, ranks U{2..16}, 1e-3 noise, "
                               "eps 1e-2", "tensors": len(xs), "elements": elems, "eps": BATCH["eps"],
                   "rmax": BATCH["rmax"],
                   "launch": "CUDA graph replay: counter/status reset, one persistent kernel (one CTA per tensor "
                             "at a time), read-back of ranks and error estimates",
                   "autotuner": {"chunk": chunk, "largest_first": largest_first,
                                 "variant_ms": {f"{'lpt' if i >= 3 else 'natural'}_chunk{c}": round(v, 3)
                                                for i, (c, v) in enumerate(zip([16, 32, 64] * 2, tune_ms))}},
                   "l2": f"inputs {elems * 4 / 1e9:.2f} GB > L2, no flush needed"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_tt_batched (whole batch, one launch)", "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": ms},
        "gpu_launches": steps, "clocks": clocks,
    }
    # parity on a sample: oracle delta-truncation ranks and the measured error of our cores
    import oracle
    sample = list(range(0, len(xs), max(1, len(xs) // 32)))
    agree, worst = 0, 0.0
    t_cpu = time.time()
    for i in sample:
        xh = xs[i].double().cpu().numpy()
        _, oranks = oracle.tt_svd_eps(xh, BATCH["eps"], max_ranks=[1] + [BATCH["rmax"]] * 3 + [1])
        agree += int(oranks == ranks[i])
        full = oracle.tt_full([c.double().cpu().numpy() for c in res[i][0]])
        worst = max(worst, oracle.rel_error(xh, full))
    t_cpu = (time.time() - t_cpu) / len(sample)
    out["parity"] = {"sample": len(sample), "rank_agreement": agree, "max_rel_err": worst,
                     "max_err_estimate": float(errs.max())}
    out["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "tensors/s", "cores": blas_threads(), "kind": "port",
                           "sample": f"oracle FP64 delta-truncated TT-SVD + reconstruction on {len(sample)} "
                                     f"tensors of the batch"}
    del b, xs
    return out


def run_batch(args):
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    r = measure_batch(args, dev, args.steps, args.warmup)
    line = {"metric": r.pop("metric"), "value": r.pop("value"), "unit": r.pop("unit"), "n_gpus": 1,
            "steps": r.pop("steps"), "warmup": r.pop("warmup"), "ms_per_step": r.pop("ms"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+fp64",
            "data": "synthetic (seeded N(0,1) TT cores, modes U{8..32}, ranks U{2..16}, 1e-3 noise)", **r}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# c5: learned vs plain adaptive EDrSVD on order-6 tensors with power-law unfolding spectra
# ---------------------------------------------------------------------------------------
C5 = dict(count=4, nmin=24, nmax=40, bond=64, amin=0.5, amax=2.0, noise=1e-5, eps=1e-3, rmax=96)


def canonical_cores(n, lam, rng, iters=400):
    """Cores M_k (r_{k-1}, n_k, r_k) of a TT in canonical (Vidal) form with bond spectra lam:
    sum_i M_k[i] M_k[i]^T = diag(lam_{k-1}^2) and sum_i M_k[i]^T M_k[i] = diag(lam_k^2), found by
    alternating projections onto the two conditions.  The tensor M_1 L_1^-1 M_2 L_2^-1 ... M_d
    then has exactly lam_k as the singular values of its unfolding k."""
    cores = []
    for k in range(len(n)):
        la, lb = lam[k], lam[k + 1]
        ra, rb = la.size, lb.size
        m = rng.standard_normal((ra, n[k], rb))
        for it in range(iters):
            u, _, vt = np.linalg.svd(m.reshape(ra, -1), full_matrices=False)
            m = (la[:, None] * (u @ vt)).reshape(ra, n[k], rb)
            u, _, vt = np.linalg.svd(m.reshape(-1, rb), full_matrices=False)
            m = ((u @ vt) * lb[None, :]).reshape(ra, n[k], rb)
            if it % 25 == 24:
                a = m.reshape(ra, -1)
                if np.abs(a @ a.T - np.diag(la * la)).max() < 1e-13:
                    break
        cores.append(m)
    return cores


def c5_tensor(seed, device):
    """One order-6 c5 tensor on the device (column-major flat FP32) and its description."""
    import torch
    cfg = C5
    rng = np.random.default_rng(seed)
    n = [int(v) for v in rng.integers(cfg["nmin"], cfg["nmax"] + 1, size=6)]
    dims = [1] + [int(min(np.prod(n[:k]), np.prod(n[k:]), cfg["bond"])) for k in range(1, 6)] + [1]
    alphas, lam = [], [np.ones(1)]
    for k in range(1, 6):
        a = float(rng.uniform(cfg["amin"], cfg["amax"]))
        l_k = np.arange(1, dims[k] + 1, dtype=np.float64) ** (-a)
        lam.append(l_k / np.linalg.norm(l_k))
        alphas.append(a)
    lam.append(np.ones(1))
    cores = canonical_cores(n, lam, rng)
    # left-canonical cores A_k = M_k L_k^-1 (k < d), contracted right to left in the column-major
    # chain layout (row-major transposes, as in clean_tensor_torch)
    mt = torch.from_numpy(cores[5][:, :, 0].T.copy()).to(device)
    for k in range(4, -1, -1):
        a_k = cores[k] / lam[k + 1][None, None, :]
        g = torch.from_numpy(np.ascontiguousarray(a_k.transpose(2, 1, 0).reshape(dims[k + 1], -1))).to(device)
        mt = (mt @ g).reshape(-1, dims[k])
    x = mt.reshape(-1).float()
    del mt
    gen = torch.Generator(device=device).manual_seed(seed + 1)
    nrm = torch.linalg.vector_norm(x.double()).item()
    x.add_(torch.randn(x.shape, generator=gen, device=device), alpha=cfg["noise"] * nrm / np.sqrt(x.numel()))
    return x, n, alphas


def measure_c5(args, dev):
    """Learned (probe -> predicted sketch width and power count, tensor-core passes, probe-based
    a-posteriori estimate) against plain adaptive EDrSVD (sketch width doubling from 16 + s,
    p = 1, exact energies) on order-6 tensors with modes U{24..40} whose unfolding spectra are
    power laws i^-alpha, alpha ~ U[0.5, 2] (bond dimension 64, 1e-5 noise), eps = 1e-3."""
    import ctypes as C
    import torch
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib, learned as _learned
    cfg = C5
    stream = torch.cuda.current_stream(dev)
    ctx = ttr._ctx_for(dev.index or 0, stream)
    ttr.set_predictor(_learned.load_params(), device=dev)
    rows = []
    try:
        for t in range(cfg["count"]):
            x, n, alphas = c5_tensor(args.seed + 101 * t, dev)
            d = 6
            maxr = [1] + [cfg["rmax"]] * (d - 1) + [1]
            row = {"n": n, "alpha": [round(a, 3) for a in alphas]}
            for name, flags in (("plain", _lib.TT_FLAG_ADAPTIVE_KS), ("learned", _lib.TT_FLAG_LEARNED)):
                o = ttr._opts("auto", "edrsvd", 8, 1, args.seed, flags, 40)
                o.eps = cfg["eps"]
                flat = [torch.empty(maxr[k] * n[k] * maxr[k + 1], device=dev) for k in range(d)]
                ptrs = (C.c_void_p * d)(*[f.data_ptr() for f in flat])
                fn = ttr.lib().tt_svd
                st = _lib.TTStats()

                def run():
                    _lib.check(fn(ctx, C.c_void_p(x.data_ptr()), d, _lib.int_array(n), _lib.int_array(maxr),
                                  C.byref(o), ptrs, C.byref(st)))
                run()
                torch.cuda.synchronize(dev)
                ms = []
                for _ in range(3):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    run()
                    e1.record(stream)
                    torch.cuda.synchronize(dev)
                    ms.append(e0.elapsed_time(e1))
                rr = list(st.ranks[: d + 1])
                err = C.c_double()
                _lib.check(ttr.lib().tt_rel_error(ctx, C.c_void_p(x.data_ptr()), d, _lib.int_array(n),
                                                  _lib.int_array(rr), 0, ptrs, C.byref(err)))
                row[name] = {"ms": float(np.median(ms)), "passes": int(st.passes), "fallbacks": int(st.fallbacks),
                             "ranks": rr, "step_ks": list(st.step_ks[: d - 1]),
                             "step_power": list(st.step_power[: d - 1]), "est_rel_err": float(st.est_rel_err),
                             "rel_err": float(err.value), "eps_unmet": int(st.eps_unmet)}
                del flat
            rows.append(row)
            del x
            torch.cuda.empty_cache()
    finally:
        ttr.set_predictor(None, device=dev)
    ok = [r for r in rows if r["plain"]["rel_err"] <= cfg["eps"] and r["learned"]["rel_err"] <= cfg["eps"]]
    out = {
        "config": {"workload": "c5: order-6 TT tensors in canonical form, modes U{24..40}, unfolding spectra "
                               "i^-alpha (alpha ~ U[0.5, 2], bond 64), 1e-5 noise, eps 1e-3, rank bound 96",
                   "tensors": cfg["count"]},
        "ms_plain": float(sum(r["plain"]["ms"] for r in rows)),
        "ms_learned": float(sum(r["learned"]["ms"] for r in rows)),
        "passes_plain": int(sum(r["plain"]["passes"] for r in rows)),
        "passes_learned": int(sum(r["learned"]["passes"] for r in rows)),
        "fallbacks": int(sum(r["learned"]["fallbacks"] for r in rows)),
        "both_meet_eps": len(ok),
        "max_rel_err": {"plain": max(r["plain"]["rel_err"] for r in rows),
                        "learned": max(r["learned"]["rel_err"] for r in rows)},
        "rows": rows,
    }
    out["learned_speedup"] = out["ms_plain"] / out["ms_learned"] if out["ms_learned"] > 0 else None
    return out


def run_reference(args, wl):
    """The reference arm: the reference's own chain for this workload restated in NumPy FP32,
    run full size on the host cores with all BLAS threads (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    xh = host_tensor(wl, args.seed)
    s, p = wl_sp(wl, args)
    gemm = args.gemm if args.gemm is not None else wl.get("gemm", "auto")
    fl = chain_flops(wl["shape"], wl["ranks"], wl["ring"], s, p, gemm)
    for _ in range(min(args.warmup, 2)):
        cpu_chain(xh, wl, s, p)
    ts = []
    t_start = time.perf_counter()
    for _ in range(args.steps):
        ts.append(cpu_chain(xh, wl, s, p))
        if time.perf_counter() - t_start > args.ref_budget:
            break
    t = float(np.mean(ts))
    cores = blas_threads()
    val = fl / t / 1e12
    algo = "plain EDrSVD chain (EDR:329-586)" if len(wl["shape"]) == 3 else \
        ("order-6 Gram-eigen TR chain (TR6:827-1004)" if wl["ring"] else "order-6 Gram-eigen TT chain (TT6:799-958)")
    sample = f"full-size {algo} in NumPy FP32 on the host cores; {len(ts)} of {args.steps} steps timed " \
             f"(time budget {args.ref_budget:.0f} s), {min(args.warmup, 2)} untimed"
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": len(ts), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["desc"], "parallelism": "host threads", "flops_per_step": fl,
                   "flops": "the GPU arm's chain FLOPs (same numerator for both arms)"},
        "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _roofline(stats, ms_step, steps, workload_key, use_traffic):
    kinds = _lib_mod().PASS_NAMES
    pass_ms = np.zeros(4)
    pass_b = np.zeros(4)
    pass_n = np.zeros(4)
    for st in stats:
        for k in range(4):
            pass_ms[k] += st.pass_ms[k]
            pass_b[k] += st.pass_bytes[k]
            pass_n[k] += st.pass_launches[k]
    # The dominant kernel: the longest single bulk pass of the chain (same pass in every step),
    # timed by CUDA events on the library's stream inside the timed region.
    top_kind, top_step = int(stats[-1].top_kind), int(stats[-1].top_step)
    top_ms = float(np.mean([st.top_ms for st in stats]))
    top_bytes = float(stats[-1].top_bytes)
    achieved = top_bytes / (top_ms * 1e-3) / 1e9
    peak, peak_src = peaks()
    key = f"{kinds[top_kind]}:{top_step}"
    n = len(stats)
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": committed_traffic(workload_key, key) if use_traffic else None,
            "kernel": f"{kinds[top_kind]} pass of unfolding {top_step + 1}", "peak_source": peak_src,
            "algorithmic_bytes_per_launch": top_bytes, "avg_launch_ms": top_ms,
            "share_of_step": float(top_ms / ms_step),
            "step_bytes_frac": float(stats[-1].bytes / (ms_step * 1e-3) / 1e9 / peak),
            "passes": {kinds[k]: {"ms": pass_ms[k] / n, "launches": pass_n[k] / n,
                                  "GBps": (pass_b[k] / (pass_ms[k] * 1e-3) / 1e9) if pass_ms[k] > 0 else None}
                       for k in range(4)}}


def _lib_mod():
    from tensor_train_ring_decompositions_hpc_gpu_b200 import _lib
    return _lib


def flush_l2(buf):
    buf.add_(1.0)  # a read + write of a buffer larger than the 126 MB L2


def measure_chain(name, wl, args, dev, local, world, steps, warmup, seed, forms=False, e2e_steps=3,
                  parity_key=None):
    """Time the fixed-rank decomposition of one workload through the C ABI (device-resident
    input, CUDA events on the library's stream, max over ranks) and collect accuracy, parity,
    roofline, end-to-end time and, on request, the other forms on the same tensor."""
    import ctypes as C
    import torch
    import torch.distributed as dist
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr
    _lib = _lib_mod()
    shape, ranks, ring = wl["shape"], wl["ranks"], wl["ring"]
    s_ov, p_pw = wl_sp(wl, args)
    gemm = args.gemm if args.gemm is not None else wl.get("gemm", "auto")
    d = len(shape)
    x = make_tensor_torch(wl, seed, dev)
    flat = [torch.empty(ranks[k] * shape[k] * ranks[k + 1], device=dev) for k in range(d)]
    ptrs = (C.c_void_p * d)(*[t.data_ptr() for t in flat])
    o = ttr._opts(gemm, "edrsvd", s_ov, p_pw, args.seed, 0, 40)
    n_arr, r_arr = _lib.int_array(shape), _lib.int_array(ranks)
    fn = ttr.lib().tr_svd if ring else ttr.lib().tt_svd
    stream = torch.cuda.current_stream(dev)
    ctx = ttr._ctx_for(local, stream)
    l2buf = torch.empty(64 << 20, dtype=torch.float32, device=dev) if wl.get("flush_l2") else None

    def step(flags=0, opts=None):
        op = opts or o
        op.flags = _lib.TT_FLAG_KEEP_SIGMA | flags | (op.flags & (_lib.TT_FLAG_LEARNED | _lib.TT_FLAG_ADAPTIVE_KS))
        st = _lib.TTStats()
        _lib.check(fn(ctx, C.c_void_p(x.data_ptr()), d, n_arr, r_arr, C.byref(op), ptrs, C.byref(st)))
        return st

    def timed_loop(nsteps, flags=0, opts=None):
        """Device ms per step; with an L2 flush between steps each step is timed alone."""
        sts = []
        if l2buf is None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(nsteps):
                sts.append(step(flags, opts))
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1) / nsteps, sts
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        for a, b in evs:
            flush_l2(l2buf)
            a.record(stream)
            sts.append(step(flags, opts))
            b.record(stream)
        torch.cuda.synchronize(dev)
        return float(np.sum([a.elapsed_time(b) for a, b in evs])) / nsteps, sts

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms, stats = timed_loop(steps, _lib.TT_FLAG_PROFILE)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())

    def rel_err_of(rr):
        e = C.c_double()
        _lib.check(ttr.lib().tt_rel_error(ctx, C.c_void_p(x.data_ptr()), d, n_arr, _lib.int_array(rr),
                                          1 if ring else 0, (C.c_void_p * d)(*[t.data_ptr() for t in flat]),
                                          C.byref(e)))
        return e.value

    err = rel_err_of(list(ranks))
    fl = chain_flops(shape, ranks, ring, s_ov, p_pw, gemm)
    lib_fl = float(stats[-1].flops)
    out = {
        "ms": ms_max, "value": fl * world / (ms_max * 1e-3) / 1e12, "unit": "TFLOP/s", "rel_err": err,
        "config": {"workload": wl["desc"], "gemm": gemm, "oversample": s_ov, "power_iters": p_pw,
                   "l2": ("L2 flushed (256 MB write) before every step, each step timed alone"
                          if l2buf is not None else
                          f"input {x.numel() * 4 / 1e9:.2f} GB > L2, no flush needed"),
                   "flops_per_step": fl, "library_flops_per_step": lib_fl,
                   "hbm_bytes_per_step": float(stats[-1].bytes)},
        "parity": exact_chain_parity(parity_key or name, seed, wl, err, stats[-1]),
        "jacobi_sweeps_max": int(max(st.jacobi_sweeps for st in stats)),
        "roofline": _roofline(stats, ms, steps, name, use_traffic=not wl.get("override")),
        "gpu_launches": int(sum(st.kernels for st in stats)), "steps": steps, "clocks": clk,
    }
    if abs(fl - lib_fl) > 1e-6 * lib_fl:
        out["config"]["flops_mismatch"] = "chain_flops differs from the library's count"

    # end to end through the public API with pinned host buffers
    if e2e_steps > 0:
        xh = torch.empty(x.numel(), dtype=torch.float32, pin_memory=True)
        xh.copy_(x)
        hc = [torch.empty(ranks[k] * shape[k] * ranks[k + 1], dtype=torch.float32, pin_memory=True)
              for k in range(d)]
        hptr = (C.c_void_p * d)(*[t.data_ptr() for t in hc])

        def hstep():
            o.flags = _lib.TT_FLAG_KEEP_SIGMA | _lib.TT_FLAG_HOST_IO
            st = _lib.TTStats()
            _lib.check(fn(ctx, C.c_void_p(xh.data_ptr()), d, n_arr, r_arr, C.byref(o), hptr, C.byref(st)))

        hstep()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        h0 = torch.cuda.Event(enable_timing=True)
        h1 = torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(e2e_steps):
            hstep()
        h1.record(stream)
        torch.cuda.synchronize(dev)
        ems = h0.elapsed_time(h1) / e2e_steps
        et = torch.tensor([ems], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        ems = float(et.item())
        out["e2e"] = {"value": fl * world / (ems * 1e-3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ems,
                      "h2d_bytes_per_step": int(x.numel() * 4),
                      "d2h_bytes_per_step": int(sum(t.numel() * 4 for t in hc)), "steps": e2e_steps}
        del xh, hc

    # The forms of one decomposition on the same tensor and GPU, every engine at the same (s, p):
    # the plain FP32 form (FP32 CUDA-core GEMMs, the reference's EDrSVD defaults s = 8, p = 1),
    # the tensor-core form at p = 0 and 1, and the learned form (eps = 1e-3, the caller's ranks
    # as bounds, the shipped predictor choosing sketch width and power count per randomized step).
    if forms:
        def form(gemm_f, p_f, flags=0, eps=0.0):
            op = ttr._opts(gemm_f, "edrsvd", s_ov, p_f, args.seed, flags, 40)
            op.eps = eps
            step(0, op)
            torch.cuda.synchronize(dev)
            f_ms, sts = timed_loop(3, 0, op)
            rr = list(sts[-1].ranks[: d + 1])
            return {"ms": f_ms, "rel_err": rel_err_of(rr), "ranks": rr, "passes": int(sts[-1].passes),
                    "step_ks": list(sts[-1].step_ks[: d - 1]), "step_power": list(sts[-1].step_power[: d - 1])}
        fm = {}
        for p_f in (0, 1):
            fm[f"tc_p{p_f}"] = form("tc", p_f)
            fm[f"tc_p{p_f}"]["config"] = f"TF32 tensor cores, fixed ranks, s = {s_ov}, p = {p_f}"
            fm[f"plain_fp32_p{p_f}"] = form("fp32", p_f)
            fm[f"plain_fp32_p{p_f}"]["config"] = f"FP32 CUDA-core GEMMs, fixed ranks, s = {s_ov}, p = {p_f}"
        fm["engine_speedup_same_s_p"] = {f"p{p_f}": fm[f"plain_fp32_p{p_f}"]["ms"] / fm[f"tc_p{p_f}"]["ms"]
                                         for p_f in (0, 1)}
        if not ring:
            from tensor_train_ring_decompositions_hpc_gpu_b200 import learned as _learned
            ttr.set_predictor(_learned.load_params(), device=dev)
            fm["learned"] = form(gemm, 1, _lib.TT_FLAG_LEARNED, 1e-3)
            fm["learned"]["config"] = ("tensor cores, eps = 1e-3 (ranks <= 32), shipped predictor choosing s and p "
                                       "per randomized step, plain adaptive EDrSVD (p = 1) as fallback")
            ttr.set_predictor(None, device=dev)
            fm["learned_speedup_vs_plain_fp32"] = fm["plain_fp32_p1"]["ms"] / fm["learned"]["ms"]
        out["forms"] = fm
    out["_x"] = x
    return out


def run_ours(args, wl):
    import torch
    import torch.distributed as dist
    import tensor_train_ring_decompositions_hpc_gpu_b200 as ttr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    ttr.lib()  # fails loudly without the built library
    head = measure_chain(args.workload, wl, args, dev, local, world, args.steps, args.warmup, args.seed + rank,
                         forms=not args.no_forms, e2e_steps=args.e2e_steps, parity_key=args.workload)
    x = head.pop("_x")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        xh = x.cpu().numpy()
        t, n = cpu_baseline(xh, wl, args, args.cpu_steps)
        cpu = {"value": head["config"]["flops_per_step"] / t / 1e12, "unit": "TFLOP/s", "cores": blas_threads(),
               "kind": "port", "ms_per_step": t * 1e3,
               "sample": f"full-size reference chain in NumPy FP32 on the same tensor, {n} steps timed after "
                         f"one untimed"}
        del xh
    del x
    torch.cuda.empty_cache()
    workloads = None
    if world == 1 and not args.no_workloads:
        workloads = run_workloads(args, dev, local)
    if rank == 0:
        c = head["config"]
        c["parallelism"] = f"replicas x{world}"
        line = {
            "metric": METRIC, "value": head["value"], "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "tf32-tc+fp32+fp64" if c["gemm"] != "fp32" else "fp32+fp64",
            "data": "synthetic (seeded random TT/TR cores + Gaussian noise)", "config": c,
            "rel_err": head["rel_err"], "parity": head["parity"], "jacobi_sweeps_max": head["jacobi_sweeps_max"],
            "roofline": head["roofline"], "forms": head.get("forms"), "cpu_baseline": cpu, "e2e": head.get("e2e"),
            "gpu_launches": head["gpu_launches"], "clocks": head["clocks"], "workloads": workloads,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_workloads(args, dev, local):
    """The other configurations, each measured in this run: timing, accuracy, parity, roofline,
    CPU baseline and end-to-end time."""
    import torch
    res = {}
    for name in args.workloads.split(","):
        if not name or name == args.workload:
            continue
        t0 = time.time()
        try:
            if name == "batch4":
                res[name] = measure_batch(args, dev)
            elif name == "c5":
                res[name] = measure_c5(args, dev)
            else:
                wl = dict(WORKLOADS[name])
                sub = argparse.Namespace(**vars(args))
                sub.oversample = None
                sub.power_iters = None
                sub.gemm = None
                r = measure_chain(name, wl, sub, dev, local, 1, min(args.steps, 10), 3, args.seed,
                                  forms=False, e2e_steps=2, parity_key=name)
                x = r.pop("_x")
                if not args.no_cpu_baseline:
                    xh = x.cpu().numpy()
                    t, n = cpu_baseline(xh, wl, sub, 2 if name != "tt3" else 10)
                    r["cpu_baseline"] = {"value": r["config"]["flops_per_step"] / t / 1e12, "unit": "TFLOP/s",
                                         "cores": blas_threads(), "kind": "port", "ms_per_step": t * 1e3,
                                         "sample": f"full-size reference chain in NumPy FP32 on the same tensor, "
                                                   f"{n} steps timed after one untimed"}
                    del xh
                del x
                res[name] = r
        except Exception as e:  # keep the headline line even if one sub-workload fails
            res[name] = {"error": f"{type(e).__name__}: {e}"}
        res.get(name, {})["wall_s"] = time.time() - t0
        torch.cuda.empty_cache()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tt6", choices=sorted(WORKLOADS) + ["batch4"])
    ap.add_argument("--batch-count", type=int, default=None,
                    help="batch4: tensors in the batch (default 4096; smaller for profiling captures)")
    ap.add_argument("--workloads", default="tt3,tr6,batch4,c5",
                    help="other configurations measured in the same run (comma list; '' for none)")
    ap.add_argument("--no-workloads", action="store_true")
    ap.add_argument("--gemm", default=None, choices=["auto", "tc", "fp32"],
                    help="engine of the headline workload (default: its configuration's)")
    ap.add_argument("--oversample", type=int, default=None,
                    help="sketch oversampling (default: the workload's, 8 for tt6 and tt3, 72 for tr6)")
    ap.add_argument("--power-iters", type=int, default=None,
                    help="power iterations (default: the workload's, 0 for tt6, 1 for tr6 and tt3)")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=2, help="full-size CPU baseline steps (after one untimed)")
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="seconds of timed CPU work in the reference arm before it stops early")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the engine and learned comparison on the same tensor")
    ap.add_argument("--shape", default=None, help="override the mode sizes, e.g. 32,32,32,32,24,24")
    ap.add_argument("--ranks", default=None, help="override the ranks, e.g. 1,32,32,32,32,24,1")
    args = ap.parse_args()
    if args.workload == "batch4":
        return run_batch(args)
    wl = dict(WORKLOADS[args.workload])
    if args.shape:
        wl["shape"] = [int(v) for v in args.shape.split(",")]
        wl["ranks"] = [int(v) for v in args.ranks.split(",")]
        wl["override"] = True
        wl["desc"] = f"{'TR' if wl['ring'] else 'TT'}-SVD of {'x'.join(map(str, wl['shape']))} " \
                     f"ranks ({','.join(map(str, wl['ranks']))}), {wl['noise']:g} noise"
    if args.impl == "reference":
        return run_reference(args, wl)
    return run_ours(args, wl)


if __name__ == "__main__":
    sys.exit(main())
