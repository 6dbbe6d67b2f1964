"""GPU tests of the plan table and the autotuner (bc_autotune, bc_plan_table_*)."""
import numpy as np
import pytest

import oracle
from conftest import raw_u64, to_dev, to_host

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_exact(gpu_ctx):
    import bc_ntt
    import torch

    bc_ntt.plan_table_clear()
    rng = np.random.default_rng(12)
    for log_n, log_b, cols in ((14, 1, 6), (17, 2, 3), (20, 0, 2), (21, 3, 2)):
        rep = bc_ntt.autotune(log_n, log_b, cols, reps=1)
        lines = rep.strip().splitlines()
        assert lines[-1].startswith("best ")
        assert len(lines) - 1 >= 8, rep  # window splits, then the launch knobs of the best one
        n = 1 << log_n
        x = raw_u64(rng, cols * n)
        if log_b:
            out = torch.empty(((1 << log_b) * cols) << log_n, dtype=torch.int64, device="cuda")
            bc_ntt.lde(to_dev(x), out, log_n, cols, log_b)
            exp = oracle.lde(x, log_n, cols, n, log_b, threads=8)
        else:
            out = torch.empty(cols * n, dtype=torch.int64, device="cuda")
            d = to_dev(x)
            bc_ntt.batch_ntt_internal(d.data_ptr(), out.data_ptr(), log_n, cols, n, n, False, False, 0, 0)
            exp = oracle.batch_ntt(x, log_n, cols, n, n, False, False, threads=8)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_host(out), exp, err_msg=f"log_n={log_n} blowup={1 << log_b}")
    bc_ntt.plan_table_clear()


def test_plan_table_roundtrip_and_validation(gpu_ctx):
    import bc_ntt

    bc_ntt.plan_table_clear()
    bc_ntt.plan_table_import("22 1 3 5 8 5 8 12 1\n16 0 2 8 8 8 1\n")
    text = bc_ntt.plan_table_export()
    assert "22 1 3 5 8 5 8 12 1" in text and "16 0 2 8 8 8 1" in text
    with pytest.raises(ValueError):
        bc_ntt.plan_table_import("22 1 2 10 4 11 1\n")  # bits do not sum to log_n
    with pytest.raises(ValueError):
        bc_ntt.plan_table_import("20 1 2 9 1 11 1\n")  # a run of 1 above bit 0
    # an imported three-pass plan is used and stays exact
    import torch

    rng = np.random.default_rng(3)
    x = raw_u64(rng, 2 << 22)
    out = torch.empty(4 << 22, dtype=torch.int64, device="cuda")
    bc_ntt.lde(to_dev(x), out, 22, 2, 1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(out), oracle.lde(x, 22, 2, 1 << 22, 1, threads=8))
    bc_ntt.plan_table_clear()
    assert bc_ntt.plan_table_export() == ""


@pytest.mark.parametrize("knobs", ["k 1 0 0 0 0", "k 32 2 0 0 0", "k 0 16 2 0 0", "k 0 0 3 0 0", "k 0 4 0 2 0",
                                   "k 0 0 0 1 3", "k 8 0 0 0 2", "k 4 2 3 2 3"])
def test_plan_knobs_stay_exact(gpu_ctx, knobs):
    """Every launch knob the autotuner may pick -- column walks, top-window table mode and double-buffering, pass
    occupancy -- gives the oracle's result, for a fused LDE with an 8-column top window (where double-buffering
    applies) and for a plain NTT."""
    import bc_ntt
    import torch

    bc_ntt.plan_table_clear()
    bc_ntt.plan_table_import(f"17 1 2 5 8 12 1 {knobs}\n17 2 2 5 8 12 1 {knobs}\n17 0 2 5 8 12 1 {knobs}\n")
    assert knobs in bc_ntt.plan_table_export()
    rng = np.random.default_rng(31)
    log_n, cols = 17, 5
    n = 1 << log_n
    x = raw_u64(rng, cols * n)
    d = to_dev(x)
    for log_b in (1, 2):
        out = torch.empty(((1 << log_b) * cols) << log_n, dtype=torch.int64, device="cuda")
        bc_ntt.lde(d, out, log_n, cols, log_b)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_host(out), oracle.lde(x, log_n, cols, n, log_b, threads=8),
                                      err_msg=f"{knobs} blowup={1 << log_b}")
    out = torch.empty(cols * n, dtype=torch.int64, device="cuda")
    bc_ntt.batch_ntt_internal(d.data_ptr(), out.data_ptr(), log_n, cols, n, n, False, False, 0, 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(out), oracle.batch_ntt(x, log_n, cols, n, n, False, False, threads=8))
    bc_ntt.plan_table_clear()


def test_plan_knobs_validation(gpu_ctx):
    import bc_ntt

    bc_ntt.plan_table_clear()
    for bad in ("17 1 2 5 8 12 1 k 0 0 4 0 0\n", "17 1 2 5 8 12 1 k 0 0 0 3 0\n", "17 1 2 5 8 12 1 k 0 0 0 0 5\n",
                "17 1 2 5 8 12 1 k 1 2 3\n"):
        with pytest.raises(ValueError):
            bc_ntt.plan_table_import(bad)
    bc_ntt.plan_table_clear()
