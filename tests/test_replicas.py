"""Multi-GPU is replicas only (every window updates the two shared tables; no data-path
collective).  bench.py combines replicas as: words of all ranks over the slowest rank's time.
This exercises that reduction with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    words, ms = bench.combine_replicas(torch, dist, 1000 * (rank + 1), 10.0 + 5.0 * rank)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (words, ms)


def test_combine_replicas_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        assert out[r] == (3000, 15.0)  # summed words, max time


def test_single_process_passthrough():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_replicas(torch, None, 123, 4.5) == (123, 4.5)
