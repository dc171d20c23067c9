"""bench.py's replica aggregation with two ranks over gloo on the CPU: the
step time is the slowest rank's, the throughput counts every rank's work."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]
        units = [1000.0, 3000.0][rank]
        out[rank] = (bench.replica_reduce(ms, "max"), bench.replica_reduce(units, "sum"))
    finally:
        dist.destroy_process_group()


def test_replica_reduce_two_ranks():
    import torch.multiprocessing as mp

    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    for r in range(2):
        assert out[r] == (20.0, 4000.0)


def test_replica_reduce_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_reduce(7.0, "max") == 7.0
    assert bench.replica_reduce(3.0, "sum") == 3.0
