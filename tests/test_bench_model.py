"""The bench's host mirror of the plan (bench.plan_steps / bench.chain_flops) on the CPU.

The FLOP totals below are the library's own pass accounting (tt_stats.flops) for the three
full-size workloads, as reported in the bench line's library_flops_per_step on a B200; the GPU
test test_bench_flop_model_matches_library checks the same identity on smaller chains.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


@pytest.mark.parametrize("name,flops", [
    ("tt6", 252293283840.0),    # 32^6 TT, ranks 32, s = 8, p = 0: folded step 1, three sketched steps
    ("tr6", 531812253696.0),    # 32^6 TR, bonds 8, s = 72, p = 1: refined exact step 2, 80-wide sketches
    ("tt3", 3700457472.0),      # 256^3 TT, ranks 16, s = 8, p = 1, FP32 engine
])
def test_chain_flops_equals_library_count(name, flops):
    wl = bench.WORKLOADS[name]
    fl = bench.chain_flops(wl["shape"], wl["ranks"], wl["ring"], wl.get("oversample", 8),
                           wl.get("power_iters", 0), wl.get("gemm", "auto"))
    assert fl == pytest.approx(flops, rel=1e-12)


def test_ring_plan_compacts_rows_and_refines_large_exact_steps():
    wl = bench.WORKLOADS["tr6"]
    steps = bench.plan_steps(wl["shape"], wl["ranks"], True, 72)
    # bond split of 64 on 32 rows: 32 kept, ceil(32 / 8) = 4 bond components carried
    assert [st["m"] for st in steps] == [32, 128, 256, 256, 256]
    assert [st["path"] for st in steps] == ["rows", "rows", "rand", "rand", "rand"]
    # the refined exact step replaces its projection (2 m n r) by Z = A^T U0, its Gram and E_r^T Z^T
    st = steps[1]
    m, n, r, b = st["m"], st["cols"], st["re"], st["re"] + 16
    with_tc = bench.chain_flops(wl["shape"], wl["ranks"], True, 72, 1, "tc")
    with_fp32 = bench.chain_flops(wl["shape"], wl["ranks"], True, 72, 1, "fp32")
    assert with_tc - with_fp32 == pytest.approx(2.0 * m * n * b + 2.0 * n * b * b + 2.0 * b * n * r
                                                - 2.0 * m * n * r, rel=1e-12)
