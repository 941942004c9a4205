"""Multi-rank aggregation of bench.py, run as two gloo ranks on the CPU.

With N GPUs the benchmark runs N independent replicas of the join (the path does not shard); the
job's time is the slowest rank's and its throughput counts every rank's tuples."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 7.0 * rank  # per-rank device time of the timed region
        worst = bench.max_over_ranks(ms, dist, "cpu")
        q.put((rank, worst, bench.whole_job_value(world, 5, 1000, 3000, worst)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_value(1, 10, 100, 300, 2000.0) == pytest.approx(2000.0)


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, worst, value in got:
        assert worst == pytest.approx(107.0)  # every rank reports the slowest rank's time
        # 2 ranks x 5 steps x 4000 tuples in 107 ms
        assert value == pytest.approx(2 * 5 * 4000 / 0.107)
