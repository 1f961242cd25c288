"""The N > 1 path of bench.py on CPU: two gloo ranks (replicas only -- QLA
has no distributed semantics) agree on the slowest rank's time and on the
whole-job rate.  No GPU involved."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        out[rank] = (ms, bench.whole_job_rate(world, 1000, 50, 2, ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1]
    ms, rate = out[0]
    assert ms == 15.0
    assert rate == pytest.approx(2 * 1000 * 50 * 2 / 0.015)


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_rate(1, 10, 5, 2, 100.0) == pytest.approx(1000.0)
