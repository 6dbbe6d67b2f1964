"""The multi-process path of bench.py on CPU: two gloo ranks on 127.0.0.1.

The LDE path does not exchange data between GPUs (columns, cosets and jobs
are independent), so `bench.py --gpus N` runs N replicas, one process per
GPU, and reports the whole job's throughput over the slowest rank's time.
This checks that reduction and the aggregation formula without a GPU.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench

    per_rank_ms = [120.0, 150.0][rank]  # rank 1 is the slow one
    bench.barrier(world)
    worst = bench.barrier_max(per_rank_ms, world)
    value = bench.whole_job_value(world, steps=4, units_per_rank_step=1_000_000, max_total_ms=worst)
    q.put((rank, worst, value))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_whole_job_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, worst, value in res:
        assert worst == pytest.approx(150.0)
        # 2 ranks x 4 steps x 1e6 units over 0.150 s
        assert value == pytest.approx(2 * 4 * 1e6 / 0.150 / 1e6)
