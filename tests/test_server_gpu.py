"""GPU tests of the continuous-batching LDE server (bc_lde_server_*).

* every request's result in a concurrent mix equals the same request run
  alone (bc_lde_fused on the device), bit for bit;
* requests larger than a slot's share of the memory budget are streamed in
  column chunks and still exact;
* host-side failure paths without any GPU fault: a wait that times out, a
  pending request that is cancelled (its output untouched), submissions that
  can never fit the budget are refused.
"""
import numpy as np
import pytest

from conftest import raw_u64, to_dev, to_host

pytestmark = pytest.mark.gpu


def _alone(x, log_n, cols, log_b):
    import bc_ntt
    import torch

    out = torch.empty(((1 << log_b) * cols) << log_n, dtype=torch.int64, device="cuda")
    bc_ntt.lde(to_dev(x), out, log_n, cols, log_b)
    torch.cuda.synchronize()
    return to_host(out)


def _pinned(a: np.ndarray):
    import torch

    return torch.from_numpy(a.view(np.int64)).pin_memory()


def test_server_mix_equals_alone(gpu_ctx):
    import bc_ntt
    import torch

    rng = np.random.default_rng(404)
    specs = [(14, 8, 1), (20, 3, 2), (16, 40, 1), (22, 2, 1), (18, 12, 2), (15, 64, 1), (21, 5, 1), (17, 9, 2),
             (19, 16, 1), (14, 200, 2), (20, 8, 1), (16, 3, 2)]
    srv = bc_ntt.LdeServer(memory_budget_bytes=3 << 30, slots=4)
    reqs = []
    for log_n, cols, log_b in specs:
        x = raw_u64(rng, cols << log_n)
        hx = _pinned(x)
        hout = torch.zeros(((1 << log_b) * cols) << log_n, dtype=torch.int64).pin_memory()
        rid = srv.submit(hx, hout, log_n, cols, log_b)
        reqs.append((rid, x, hout, log_n, cols, log_b))
    for rid, x, hout, log_n, cols, log_b in reqs:
        lat = srv.wait(rid, timeout_ms=120000)
        assert lat > 0
        np.testing.assert_array_equal(hout.numpy().view(np.uint64), _alone(x, log_n, cols, log_b),
                                      err_msg=f"log_n={log_n} cols={cols}")
    st = srv.stats()
    assert st["completed"] == len(specs) and st["pending"] == 0 and st["running"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["out_melem_per_s"] > 0
    srv.close()


def test_server_chunks_requests_bigger_than_a_slot(gpu_ctx):
    import bc_ntt
    import torch

    rng = np.random.default_rng(5)
    log_n, cols, log_b = 20, 24, 2  # 24 x 2^20 x 5 words = 960 MiB of in + out
    x = raw_u64(rng, cols << log_n)
    srv = bc_ntt.LdeServer(memory_budget_bytes=512 << 20, slots=2)  # 256 MiB per slot: 6 columns per chunk
    hout = torch.zeros(((1 << log_b) * cols) << log_n, dtype=torch.int64).pin_memory()
    rid = srv.submit(_pinned(x), hout, log_n, cols, log_b)
    srv.wait(rid)
    np.testing.assert_array_equal(hout.numpy().view(np.uint64), _alone(x, log_n, cols, log_b))
    # a request whose single column cannot fit a slot's share is refused up front
    with pytest.raises(ValueError):
        big = torch.zeros(1 << 24, dtype=torch.int64).pin_memory()
        srv.submit(big, big, 24, 1, 3)
    srv.close()


def test_server_cancel_and_timeout_paths(gpu_ctx):
    import bc_ntt
    import torch

    rng = np.random.default_rng(6)
    srv = bc_ntt.LdeServer(memory_budget_bytes=1 << 30, slots=1)
    head_x = raw_u64(rng, 64 << 20)  # a long head request keeps the single slot busy
    head_out = torch.zeros(2 * (64 << 20), dtype=torch.int64).pin_memory()
    head = srv.submit(_pinned(head_x), head_out, 20, 64, 1)
    tail_x = raw_u64(rng, 4 << 16)
    sentinel = 0x77
    tail_out = torch.full((2 * (4 << 16),), sentinel, dtype=torch.int64).pin_memory()
    tail = srv.submit(_pinned(tail_x), tail_out, 16, 4, 1)
    assert srv.cancel(tail) is True
    with pytest.raises(RuntimeError):
        srv.wait(tail, timeout_ms=1000)
    # a zero-length wait on the running head request times out on the host
    state, _ = srv.poll(head)
    if state in (bc_ntt.LdeServer.PENDING, bc_ntt.LdeServer.RUNNING):
        with pytest.raises(TimeoutError):
            srv.wait(head, timeout_ms=0)
    srv.wait(head, timeout_ms=120000)
    assert srv.cancel(head) is False  # already ran
    assert bool((tail_out == sentinel).all())  # the cancelled request never wrote its output
    np.testing.assert_array_equal(head_out.numpy().view(np.uint64), _alone(head_x, 20, 64, 1))
    # released records are forgotten; the slot and the statistics stay right
    assert srv.release(head) is True and srv.release(tail) is True
    with pytest.raises(ValueError):
        srv.poll(head)
    with pytest.raises(ValueError):
        srv.release(tail)
    again_out = torch.zeros(2 * (4 << 16), dtype=torch.int64).pin_memory()
    again = srv.submit(_pinned(tail_x), again_out, 16, 4, 1)
    srv.wait(again, timeout_ms=120000)
    assert srv.release(again) is True  # finished: its slot is retired here if the worker has not yet
    np.testing.assert_array_equal(again_out.numpy().view(np.uint64), _alone(tail_x, 16, 4, 1))
    st = srv.stats()
    assert st["completed"] == 2 and st["pending"] == 0 and st["running"] == 0
    srv.close()


@pytest.mark.parametrize("max_batch_elems", [1 << 22, 0])
def test_server_device_requests_equal_alone(gpu_ctx, max_batch_elems):
    """Requests on device buffers: small ones pending together are coalesced into one persistent batch launch
    (or, with coalescing off, each runs as its own fused LDE), big ones run alone; every result equals the same
    request computed alone, bit for bit, including when host requests are in the mix."""
    import bc_ntt
    import torch

    rng = np.random.default_rng(505)
    specs = [(10 + (i % 7), 1 + (i * 5) % 9, 1 + i % 3) for i in range(40)] + [(21, 6, 1), (19, 20, 2)]
    srv = bc_ntt.LdeServer(memory_budget_bytes=2 << 30, slots=2)
    srv.set_device_batching(max_batch_elems)
    reqs = []
    for log_n, cols, log_b in specs:
        x = raw_u64(rng, cols << log_n)
        out = torch.full((((1 << log_b) * cols) << log_n,), 7, dtype=torch.int64, device="cuda")
        reqs.append((x, out, log_n, cols, log_b))
    hx = raw_u64(rng, 8 << 16)
    hout = _pinned(np.zeros(2 * 8 << 16, dtype=np.uint64))
    ids = [srv.submit_device(to_dev(x), out, log_n, cols, log_b) for x, out, log_n, cols, log_b in reqs]
    hid = srv.submit(_pinned(hx), hout, 16, 8, 1)
    for i in ids + [hid]:
        srv.wait(i, timeout_ms=120000)
    st = srv.device_stats()
    srv.close()
    for x, out, log_n, cols, log_b in reqs:
        np.testing.assert_array_equal(to_host(out), _alone(x, log_n, cols, log_b),
                                      err_msg=f"log_n={log_n} cols={cols} B={1 << log_b}")
    np.testing.assert_array_equal(hout.numpy().view(np.uint64), _alone(hx, 16, 8, 1))
    assert st["batched_requests"] + st["single_requests"] == len(specs)
    if max_batch_elems:
        assert st["batches"] >= 1 and st["batched_requests"] >= 2
    else:
        assert st["batches"] == 0
