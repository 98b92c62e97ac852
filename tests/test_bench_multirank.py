"""The bench's multi-GPU arithmetic on CPU: two gloo ranks (127.0.0.1), each
with its own timing; the job time is the slowest rank's and the value the
weak-scaling aggregate (replicas, no data-path collective)."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(times[rank], dist, device="cpu")
        out[rank] = (ms, bench.job_value(world, 100, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, times = 2, [12.5, 20.0]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), times, out), nprocs=world, start_method="spawn")
    for r in range(world):
        ms, value = out[r]
        assert ms == max(times)
        assert value == pytest.approx(world * 100 / (max(times) / 1e3))


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.0, None) == 7.0
    assert bench.job_value(1, 50, 10.0) == pytest.approx(5000.0)
