"""The top-window kernel's direct path (era-boojum-cuda_b200/csrc/lde.cuh,
top_body_direct): every window shape that takes it (K >= 4 over runs of
C >= 4 low positions: <4..9, 8> and <10, 4>), forced through the plan table,
against the oracle's coset LDE.

Each shape runs as the top window of a two-pass plan (bottom pass 8/1), at
blowups 2 and 8, over a ragged column count, with the forward power tables
resident (default), prefetched one coset ahead, recomputed per coset, and with
a short column walk per CTA; one three-pass plan puts a 4-bit direct top window
above a 4-bit middle pass.
"""
import numpy as np
import pytest

import oracle
from conftest import raw_u64, to_dev, to_host

DIRECT_SHAPES = [(4, 8), (5, 8), (6, 8), (7, 8), (8, 8), (9, 8), (10, 4)]
# "" = built-in knobs (resident tables where they fit); then top_mode PREFETCH, REFILL; then top_walk 2
KNOBS = ("", " k 0 0 2 0 0", " k 0 0 3 0 0", " k 0 2 0 0 0")


def _run_plans(log_n, cols, passes, seed):
    import bc_ntt
    import torch

    n = 1 << log_n
    rng = np.random.default_rng(seed)
    x = raw_u64(rng, cols * n)
    d = to_dev(x)
    expected = {b: oracle.lde(x, log_n, cols, n, b, threads=8) for b in (1, 3)}
    try:
        for knobs in KNOBS:
            bc_ntt.plan_table_clear()
            bc_ntt.plan_table_import("".join(f"{log_n} {b} {passes}{knobs}\n" for b in (1, 3)))
            for log_b in (1, 3):
                out = torch.empty(((1 << log_b) * cols) << log_n, dtype=torch.int64, device="cuda")
                bc_ntt.lde(d, out, log_n, cols, log_b)
                torch.cuda.synchronize()
                np.testing.assert_array_equal(to_host(out), expected[log_b],
                                              err_msg=f"plan {passes}{knobs} blowup={1 << log_b}")
    finally:
        bc_ntt.plan_table_clear()


@pytest.mark.gpu
@pytest.mark.parametrize("K,C", DIRECT_SHAPES)
def test_direct_top_window_two_pass(gpu_ctx, K, C):
    _run_plans(K + 8, 11, f"2 {K} {C} 8 1", seed=100 + K)


@pytest.mark.gpu
def test_direct_top_window_three_pass(gpu_ctx):
    _run_plans(16, 9, "3 4 8 4 8 8 1", seed=7)
