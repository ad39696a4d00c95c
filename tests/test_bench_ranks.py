"""The bench's multi-rank logic on two gloo ranks on the CPU: replicas, barrier, max-over-ranks
timing and the whole-job value (pairs of all ranks over the slowest rank's time)."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    sys.path.insert(0, REPO)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        r = bench.Ranks(world, torch.device("cpu"))
        r.barrier()
        my_ms = 100.0 + 50.0 * rank  # rank 1 is the slowest
        value, slowest = r.value(pairs_per_rank=1000, steps=4, total_ms_this_rank=my_ms)
        out[rank] = (value, slowest, r.max(rank * 3.0))
    finally:
        dist.destroy_process_group()


def test_two_rank_value_uses_the_slowest_rank():
    port = 29500 + (os.getpid() % 1000)
    with mp.get_context("spawn").Manager() as m:  # no fork of a process that runs threads
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        value, slowest, mx = res[rank]
        assert slowest == 150.0 and mx == 3.0
        assert value == pytest.approx(1000 * 4 * 2 / 0.150)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    r = bench.Ranks(1)
    r.barrier()
    v, t = r.value(10, 2, 20.0)
    assert t == 20.0 and v == pytest.approx(10 * 2 / 0.020)
