"""GPU parity of the single-launch uneven LDE batch (bc_lde_batch_*).

Every job of a mixed batch must equal the same job run alone through
bc_lde_fused (and, for small jobs, the CPU oracle), bit for bit; the captured
graph must give identical results when replayed; the bounded dependency waits
must not have fired.
"""
import numpy as np
import pytest

import oracle
from conftest import raw_u64, to_dev, to_host, uniform

pytestmark = pytest.mark.gpu


def _mixed_jobs(rng, specs):
    import torch

    jobs = []
    for log_n, cols, log_b in specs:
        n = 1 << log_n
        x = raw_u64(rng, cols * n)
        ev = to_dev(x)
        out = torch.full(((1 << log_b) * cols * n,), 0x3C3C3C3C, dtype=torch.int64, device="cuda")
        jobs.append((ev, out, log_n, cols, log_b, x))
    return jobs


SPECS = [(1, 3, 1), (4, 5, 3), (9, 2, 2), (11, 7, 1), (12, 1, 3), (12, 9, 2), (13, 3, 1), (14, 40, 2),
         (15, 2, 3), (16, 17, 1), (17, 1, 2), (18, 5, 3), (19, 3, 1), (20, 2, 2), (21, 1, 1), (22, 3, 3)]


def test_batch_matches_fused_and_oracle(gpu_ctx):
    import bc_ntt
    import torch

    rng = np.random.default_rng(123)
    jobs = _mixed_jobs(rng, SPECS)
    plan = bc_ntt.LdeBatch([j[:5] for j in jobs])
    info = plan.info()
    assert info["records"] >= len(SPECS) and info["items"] > 0 and info["grid"] > 0
    plan.run()
    assert plan.status() == 0
    first = [to_host(j[1]).copy() for j in jobs]
    for (ev, out, log_n, cols, log_b, x), got in zip(jobs, first):
        ref = torch.empty_like(out)
        bc_ntt.lde(ev, ref, log_n, cols, log_b, fused=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got, to_host(ref), err_msg=f"log_n={log_n} cols={cols} B={1 << log_b}")
        if log_n <= 16:
            n = 1 << log_n
            np.testing.assert_array_equal(got, oracle.lde(x, log_n, cols, n, log_b, threads=4))
    # graph replay: same results, outputs rewritten from scratch
    for ev, out, *_ in jobs:
        out.fill_(0)
    plan.run()
    assert plan.status() == 0
    for (ev, out, *_), got in zip(jobs, first):
        np.testing.assert_array_equal(to_host(out), got)
    plan.close()


def test_batch_uneven_workload_sample(gpu_ctx):
    """A scaled-down draw of the 96-job uneven workload: every job equal to bc_lde_fused alone."""
    import bc_ntt
    import torch
    import workloads

    specs = workloads.uneven_batch(n_jobs=24, seed=5, max_total_bytes=12 << 30)
    tens = []
    for s in specs:
        g = torch.Generator(device="cuda").manual_seed(s.seed)
        ev = torch.randint(-(2**63), 2**63 - 1, (s.in_words,), device="cuda", dtype=torch.int64, generator=g)
        tens.append((ev, torch.empty(s.out_words, dtype=torch.int64, device="cuda"), s.log_n, s.cols, s.log_blowup))
    plan = bc_ntt.LdeBatch(tens)
    plan.run()
    assert plan.status() == 0
    for ev, out, log_n, cols, log_b in tens:
        ref = torch.empty_like(out)
        bc_ntt.lde(ev, ref, log_n, cols, log_b)
        torch.cuda.synchronize()
        assert torch.equal(out, ref), f"log_n={log_n} cols={cols}"
        del ref
    plan.close()


def test_batch_rejects_bad_jobs(gpu_ctx):
    import bc_ntt
    import torch

    x = torch.zeros(1 << 10, dtype=torch.int64, device="cuda")
    out = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):
        bc_ntt.LdeBatch([(x, out, 10, 1, 0)])
    with pytest.raises(ValueError):
        bc_ntt.LdeBatch([(x, out, 26, 1, 2)])


def test_batch_empty_and_single(gpu_ctx):
    import bc_ntt

    rng = np.random.default_rng(8)
    plan = bc_ntt.LdeBatch([])
    plan.run()
    assert plan.status() == 0
    plan.close()
    x = uniform(rng, 1 << 12)
    ev = to_dev(x)
    import torch

    out = torch.empty(2 << 12, dtype=torch.int64, device="cuda")
    plan = bc_ntt.LdeBatch([(ev, out, 12, 1, 1)])
    plan.run()
    assert plan.status() == 0
    np.testing.assert_array_equal(to_host(out), oracle.lde(x, 12, 1, 1 << 12, 1))
    plan.close()


def test_hybrid_plan_standalone_big_jobs(gpu_ctx):
    """Big jobs as their own kernels on a forked graph branch, small ones in the persistent kernel: exact."""
    import bc_ntt
    import torch

    rng = np.random.default_rng(77)
    jobs = _mixed_jobs(rng, SPECS)
    for min_ctas in (64, 1):  # a mix of both paths, then every job standalone
        for ev, out, *_ in jobs:
            out.fill_(0)
        plan = bc_ntt.LdeBatch([j[:5] for j in jobs], standalone_min_ctas=min_ctas)
        plan.run()
        assert plan.status() == 0
        for ev, out, log_n, cols, log_b, x in jobs:
            ref = torch.empty_like(out)
            bc_ntt.lde(ev, ref, log_n, cols, log_b, fused=True)
            torch.cuda.synchronize()
            assert torch.equal(out, ref), f"min_ctas={min_ctas} log_n={log_n} cols={cols}"
        plan.close()


def test_batch_wait_limit_expires_then_recovers(gpu_ctx):
    """Failure detection of the persistent kernel's dependency waits, without a GPU fault.

    One job of three dependent kernels, the first of them thousands of CTAs wide: the first work item of the
    second kernel is taken while items of the first are still running, so it must wait.  With a wait limit of
    one SM clock cycle that wait runs out: the kernel must set status bit 0, skip the item and still return
    (the status read synchronises the stream).  With the default limit restored, the next run must be exact."""
    import bc_ntt
    import torch

    rng = np.random.default_rng(99)
    jobs = _mixed_jobs(rng, [(20, 64, 1)])
    plan = bc_ntt.LdeBatch([j[:5] for j in jobs])
    assert plan.info()["records"] >= 3
    plan.set_wait_limit(1)
    plan.run()
    assert plan.status() & 1, "a one-cycle dependency wait must run out"
    torch.cuda.synchronize()
    plan.set_wait_limit(0)
    for j in jobs:
        j[1].fill_(0)
    plan.run()
    assert plan.status() == 0
    ev, out, log_n, cols, log_b, _ = jobs[0]
    ref = torch.empty_like(out)
    bc_ntt.lde(ev, ref, log_n, cols, log_b, fused=True)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    plan.close()
