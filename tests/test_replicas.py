"""bench.py's multi-GPU path is N independent replicas: the job's time is the
slowest rank's, its throughput all ranks' work over that time.  Exercised
here with two gloo ranks on the CPU."""

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = [2.0, 3.0][rank]  # rank 1 is the slow replica
        years = 1.5                 # each replica simulates the same model time
        m = bench.reduce_max(seconds, dist, "cpu")
        thr = bench.replica_throughput(years, seconds, world, dist, "cpu")
        dist.barrier()
        out[rank] = (m, thr)
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    for r in (0, 1):
        m, thr = res[r]
        assert m == 3.0
        assert thr == pytest.approx(2 * 1.5 / 3.0)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(2.5, None, "cpu") == 2.5
    assert bench.replica_throughput(1.5, 3.0, 1, None, "cpu") == pytest.approx(0.5)
