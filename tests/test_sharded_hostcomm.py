"""The per-rank (SPMD) sharded solver with two real processes.

Two processes, one z-slab each, both on cuda:0, exchange their halo planes and
sum their reductions through ``Problem.attach_torch_distributed`` over gloo
(host memory): the library runs each rank's step list exactly as it does with
NCCL, only the transport differs.  No kernel waits on the other process --
every exchange is a host-side synchronisation between launches -- so the two
ranks may share one GPU.  Results must match the oracle's restatement of the
multi-rank algorithm (SpMV and V-cycle bit-exact, CG and the mixed solver to
the oracle's iteration counts).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

pytestmark = pytest.mark.gpu

LOCAL = (16, 16, 8)
RANKS = 2


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
                            timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(0)
    from hpcg_b200 import Problem
    from oracle.oracle import Oracle
    nx, ny, nz = LOCAL
    L, _, _, _ = Oracle.slab_hierarchy(nx, ny, nz, world)
    n = L[0].nrow
    lo, hi = rank * n // world, (rank + 1) * n // world
    u = Oracle.uniform(1, n, -1.0, 1.0)
    r = Oracle.uniform(12, n)
    b = Oracle.spmv(L[0], u)
    P = Problem(nx, ny, nz, nranks=world, rank=rank)
    P.generate("hpcg")
    P.build_mixed()
    P.attach_torch_distributed()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a[lo:hi])).cuda()  # noqa: E731
    res = {"spmv": P.spmv(dev(u)).cpu().numpy(), "mg": P.mg(dev(r)).cpu().numpy()}
    for name, f in (("cg", P.cg), ("mixed", P.cg_mixed)):
        x = torch.zeros(hi - lo, dtype=torch.float64, device="cuda")
        k, nr, nr0 = f(dev(b), x, 500, 1e-10)
        res[name] = (k, nr / nr0, x.cpu().numpy())
    out[rank] = res
    dist.barrier()
    P.close()
    dist.destroy_process_group()


def test_two_processes_exchange_through_torch_distributed(oracle):
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(RANKS, port, out), nprocs=RANKS, join=True,
                       start_method="spawn")
    nx, ny, nz = LOCAL
    L, _, _, _ = oracle.slab_hierarchy(nx, ny, nz, RANKS)
    oracle.colour_order(L)
    n = L[0].nrow
    u = oracle.uniform(1, n, -1.0, 1.0)
    r = oracle.uniform(12, n)
    b = oracle.spmv(L[0], u)
    cat = lambda key: np.concatenate([out[k][key] for k in range(RANKS)])  # noqa: E731
    assert (cat("spmv") == b).all()
    assert (cat("mg") == oracle.mg(L, r, coloured=True)).all()
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 500, 1e-10, precond=True, coloured=True)
    for k in range(RANKS):
        assert out[k]["cg"][0] == ok and out[k]["cg"][1] <= 1e-10
    x = np.concatenate([out[k]["cg"][2] for k in range(RANKS)])
    assert np.abs(x - ox).max() <= 1e-8 * np.abs(ox).max()
    fx, fk, fnr, fnr0 = oracle.fcg(L, b, np.zeros(n), 500, 1e-10)
    for k in range(RANKS):
        assert out[k]["mixed"][0] == fk and out[k]["mixed"][1] <= 1e-10


def _slow_peer(rank, out):
    """One rank whose sum function queues ~2 s of unrelated GPU work on the
    library's stream the first time it runs: the per-iteration wait (limit
    0.5 s) must give up with ETIMEOUT, and the problem must work again once the
    queued work has drained."""
    import sys
    os.environ["HPCGX_WAIT_TIMEOUT_S"] = "0.5"
    sys.path.insert(0, ROOT)
    torch.cuda.set_device(0)
    from hpcg_b200 import HPCGXError, Problem
    P = Problem(16, 16, 16)
    P.generate("hpcg")
    n = P.rows()
    b = P.spmv(torch.ones(n, dtype=torch.float64, device="cuda"))
    # few long launches (the launch queue of a stream is short: thousands of
    # small ones would block the enqueueing host instead of the GPU)
    a = torch.randn(16384, 16384, dtype=torch.bfloat16, device="cuda")
    state = {"slow": True}

    def halo(slo, rlo, shi, rhi, count, esize, stream):
        pass                                   # one rank: never called

    def sum_(buf, count, stream):
        if state["slow"]:
            state["slow"] = False
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                for _ in range(300):
                    a @ a

    P.attach_comm(halo, sum_)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    try:
        P.cg(b, x, 50, 1e-10)
        out["code"] = 0
    except HPCGXError as e:
        out["code"] = e.code
    torch.cuda.synchronize()
    x.zero_()
    k, nr, nr0 = P.cg(b, x, 50, 1e-10)
    out["after"] = (k, nr / nr0)
    P.close()


def test_bounded_wait_reports_a_stalled_rank():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_slow_peer, args=(out,), nprocs=1, join=True, start_method="spawn")
    assert out["code"] == 8                     # HPCGX_ETIMEOUT
    k, rel = out["after"]
    assert rel <= 1e-10
