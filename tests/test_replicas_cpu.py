"""Multi-GPU runs are independent replicas (the solve does not shard): the only
collective is the timing reduction of bench.py.  Exercised here with two gloo
ranks on the CPU."""
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


def _rank(rank, world, port, times, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        total = bench.replica_time(times[rank], world)
        out[rank] = bench.per_solve_ms(total, 10, world)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replica_timing_is_max_over_ranks(world):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    times = [123.0, 456.0][:world]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time; 10 solves per rank
    for r in range(world):
        assert out[r] == pytest.approx(max(times) / (10 * world))


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_time(5.0, 1) == 5.0
    assert bench.per_solve_ms(50.0, 10, 1) == 5.0
