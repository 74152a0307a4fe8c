"""bench.py's job figures over replicas, on CPU: two gloo ranks each report
their own times and work; every rank must get the slowest rank's times and
the sum of the work (the value a multi-GPU run prints)."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r: times 10 + r and 20 - r ms, work 1000 (r + 1) and 7 (r + 1)
        got = bench.combine_ranks(dist, 10.0 + rank, 20.0 - rank, 1000 * (rank + 1), 7 * (rank + 1), "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_two_replicas_combine_to_slowest_time_and_summed_work():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(rank_main, args=(world, free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, e2e_ms, ps, e2e = out[r]
        assert (ms, e2e_ms) == (11.0, 20.0)
        assert (ps, e2e) == (3000.0, 21.0)


def test_one_process_passes_its_figures_through():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.combine_ranks(None, 5.0, 6.0, 7, 8, "cpu") == (5.0, 6.0, 7.0, 8.0)
