"""bench.py's multi-process path (replicas, one rank per GPU) on CPU: two
gloo ranks combine their timings and work exactly as the NCCL ranks do --
the slowest rank's times, the sum of every rank's processed edges -- and the
reference arm runs on rank 0 only."""

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
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: device time 10 + r ms, e2e 2 + r s, 1000 * (r + 1) edges, 7 * (r + 1) e2e edges
        got = bench.combine_replicas(dist, "cpu", 10.0 + rank, 2.0 + rank, 1000 * (rank + 1), 7 * (rank + 1))
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_combine_max_time_sum_work():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    for r in range(world):
        assert res[r] == (11.0, 3.0, 3000.0, 21.0)


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.combine_replicas(None, "cpu", 5, 1.5, 10, 4) == (5.0, 1.5, 10.0, 4.0)


def test_reference_arm_is_rank0_only(capsys):
    """Under torchrun the reference arm runs on rank 0; other ranks exit
    without work or output."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(steps=1, warmup=0, workload="rmat22_pagerank")
    bench.run_reference(args, rank=1, world=2)
    assert capsys.readouterr().out == ""
