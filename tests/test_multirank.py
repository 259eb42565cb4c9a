"""Host logic of bench.py's multi-GPU mode on CPU ranks (gloo, world size 2):
the reported time is the max over ranks and global norms sum the ranks'
squares.  No GPU is needed."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    import bench
    vals = [1.0 + rank, 10.0 - rank, 0.5 * rank]
    got = bench.max_over_ranks(vals, dist)
    tot = bench.sum_over_ranks(vals, dist)
    dist.barrier()
    out[rank] = (got, tot)
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1] == ([2.0, 10.0, 0.5], [3.0, 19.0, 0.5])


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench.sum_over_ranks([3.0, 4.0]) == [3.0, 4.0]
