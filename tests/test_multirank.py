"""The multi-GPU bench path on CPU: ranks are independent replicas whose
times combine as the slowest rank's (max over ranks) and whose throughput
is every rank's work over that time; the reference arm runs on rank 0 only.
Two gloo ranks on 127.0.0.1 stand in for two GPUs."""
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


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = bench.max_over_ranks([10.0 * (rank + 1), 100.0 - rank])
        out[rank] = (times, bench.job_rate(3, world, times[0]))
        # the reference arm: every rank other than 0 returns at once, printing nothing
        if rank != 0:
            class A:
                steps, warmup = 1, 0
            assert bench.run_reference(A()) is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        times, rate = res[rank]
        assert times == [20.0, 100.0]           # max over ranks, per value
        assert rate == pytest.approx(3 * 2 / 0.020)  # both ranks' solves over the slowest time


def test_single_process_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert bench.job_rate(6, 1, 1000.0) == pytest.approx(6.0)
