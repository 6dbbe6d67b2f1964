"""The batch entry point that allocates nothing (bc_lde_batch_noalloc).

It exists for callers that cannot call cudaMalloc -- a prover whose own pool
already holds nearly all of device memory, or a submission path that must not
trigger cudaMalloc's device-wide synchronisation -- and keeps its schedule in
a fixed array inside the library.  Its output must equal the existing
bc_lde_fused entry point, bit for bit, on two calls in a row (the second call
reuses the array the first one left behind).  This file is collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import raw_u64, to_dev, to_host

pytestmark = pytest.mark.gpu

SPECS_A = [(3, 2, 1), (12, 3, 2), (13, 1, 1), (16, 5, 3), (18, 2, 1), (20, 1, 2)]
SPECS_B = [(10, 4, 3), (14, 7, 1), (17, 3, 2), (21, 2, 1)]


def _jobs(rng, specs):
    import torch

    import bc_ntt

    out = []
    for log_n, cols, log_b in specs:
        n = 1 << log_n
        ev = to_dev(raw_u64(rng, cols * n))
        dst = torch.full(((1 << log_b) * cols * n,), 0x11, dtype=torch.int64, device="cuda")
        out.append((ev, dst, log_n, cols, log_b))
    arr = (bc_ntt.LdeJob * len(out))()
    for i, (ev, dst, log_n, cols, log_b) in enumerate(out):
        n = 1 << log_n
        arr[i] = bc_ntt.LdeJob(ev.data_ptr(), dst.data_ptr(), n, n, cols * n, log_n, cols, log_b, 0)
    return out, arr


def _run_noalloc(arr, n):
    import torch

    import bc_ntt

    status = ctypes.c_uint32(0xFFFF)
    rc = bc_ntt.lib().bc_lde_batch_noalloc(ctypes.cast(arr, ctypes.c_void_p), n,
                                           torch.cuda.current_stream().cuda_stream, ctypes.byref(status))
    assert rc == 0, f"bc_lde_batch_noalloc returned {rc}"
    assert status.value == 0


def _check_against_fused(jobs):
    import torch

    import bc_ntt

    for ev, dst, log_n, cols, log_b in jobs:
        ref = torch.empty_like(dst)
        bc_ntt.lde(ev, ref, log_n, cols, log_b, fused=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_host(dst), to_host(ref), err_msg=f"log_n={log_n} cols={cols}")


def test_noalloc_batch_matches_fused_twice(gpu_ctx):
    rng = np.random.default_rng(2025)
    jobs_a, arr_a = _jobs(rng, SPECS_A)
    _run_noalloc(arr_a, len(SPECS_A))
    _check_against_fused(jobs_a)
    # second call in a row, different jobs: the array still holds the first schedule
    jobs_b, arr_b = _jobs(rng, SPECS_B)
    _run_noalloc(arr_b, len(SPECS_B))
    _check_against_fused(jobs_b)


def test_noalloc_batch_rejects_oversized_schedule(gpu_ctx):
    import torch

    import bc_ntt

    # one job whose schedule needs far more than the fixed array: 2^24 x 4096 columns (pointers are never touched)
    big = (bc_ntt.LdeJob * 1)()
    big[0] = bc_ntt.LdeJob(16, 16, 1 << 24, 1 << 24, 4096 << 24, 24, 4096, 1, 0)
    rc = bc_ntt.lib().bc_lde_batch_noalloc(ctypes.cast(big, ctypes.c_void_p), 1,
                                           torch.cuda.current_stream().cuda_stream, None)
    assert rc == 1  # cudaErrorInvalidValue


def test_noalloc_batch_rejects_stream_capture(gpu_ctx):
    """Its schedule is copied from host memory the call frees on return, so a call on a capturing stream is
    refused (cudaErrorStreamCaptureUnsupported) and enqueues nothing; the stream stays usable afterwards."""
    import torch

    import bc_ntt

    rng = np.random.default_rng(7)
    jobs, arr = _jobs(rng, [(12, 2, 1)])
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(graph, stream=side):
        rcs.append(bc_ntt.lib().bc_lde_batch_noalloc(ctypes.cast(arr, ctypes.c_void_p), 1, side.cuda_stream, None))
    assert rcs == [900]  # cudaErrorStreamCaptureUnsupported
    del graph
    _run_noalloc(arr, 1)
    _check_against_fused(jobs)
