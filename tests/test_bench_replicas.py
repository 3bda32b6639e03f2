"""bench.py's replica timing across ranks, as world-size-2 gloo process groups
on the CPU: every rank gets the slowest rank's time, and the whole-job
throughput counts the solves of all replicas over that time."""
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times_ms, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(times_ms[rank], world, "cpu")
        out[rank] = (slowest, bench.replica_throughput(10, world, slowest))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    times = [250.0, 400.0]
    mp.start_processes(_rank_main, args=(2, _free_port(), times, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 400.0
    # 2 replicas x 10 solves in 0.4 s
    assert abs(out[0][1] - 50.0) < 1e-12 and out[0][1] == out[1][1]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(123.5, 1, "cpu") == 123.5
    assert bench.replica_throughput(10, 1, 500.0) == 20.0
