"""bench.py's multi-process bookkeeping on CPU (world size 2, gloo): each
rank's timings reduce to the maximum over the ranks on every rank, and the
whole-job rate counts every replica's product per step at the slowest rank's
time.  The product path itself has no exchange between ranks (replicas)."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import bench  # noqa: E402


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = [1.0 + rank, 10.0 - rank, 5.0]
    out[rank] = bench.max_over_ranks(torch, dist, mine, torch.device("cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_processes():
    world, port = 2, 29533 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
        got = dict(out)
    assert got[0] == got[1] == [2.0, 10.0, 5.0]


def test_job_rate_counts_every_replica():
    assert bench.job_rate(1, 0.25) == pytest.approx(4000.0)
    assert bench.job_rate(4, 0.5) == pytest.approx(8000.0)
