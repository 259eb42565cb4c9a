"""The sharded (z-slab) algorithm on CPU ranks (gloo, world sizes 2 and 3:
edge ranks with one neighbour, and an interior rank with two).

Each rank does what the reference's MPI build does on a 1 x 1 x 2 process
grid: it holds only its own slab (rows with local numbering, columns of the
neighbouring slab pointing into halo planes), exchanges the boundary planes
before every SpMV and every SYMGS (src/ExchangeHalo.cpp:34-110 as called from
src/ComputeSPMV_ref.cpp:55 and src/ComputeSYMGS_ref.cpp:56), runs the
oracle's restatements of the _ref kernels on its rows, and sums dot products
with an all-reduce (src/ComputeDotProduct_ref.cpp:66-77).  The results must
equal, bit for bit, the oracle's global restatement of the same algorithm
(Oracle.slab_hierarchy: block-Jacobi SYMGS with the other slabs' values
frozen at the start of each sweep, per-slab dot products summed in rank
order), which the GPU group is tested against.  The library's order of the
V-cycle on a slab (restriction and prolongation fused into the sweeps, two
one-plane fix-ups around the exchanges) is restated too and must give the
reference order's result.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

LOCAL = (16, 8, 8)      # nx, ny, nz per rank


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _Slab:
    """Rank r's part of one level: local rows, columns into [lower halo | rows | upper halo]."""

    def __init__(self, lev, r, nx, ny, nz):
        self.S = nx * ny * nz
        self.plane = nx * ny
        lo, hi = r * self.S, (r + 1) * self.S
        self.nnz = np.ascontiguousarray(lev.nnz[lo:hi])
        self.cols = np.ascontiguousarray(lev.cols[lo * 27:hi * 27] - lo).astype(np.int32)
        self.vals = np.ascontiguousarray(lev.vals[lo * 27:hi * 27])
        self.diag = np.ascontiguousarray(lev.diag[lo:hi])
        order = lev.order[(lev.order >= lo) & (lev.order < hi)] - lo
        self.order = np.ascontiguousarray(order.astype(np.int64))
        self.f2c = None
        self.r = r

    def ext(self, v=None):
        """A vector with one halo plane on each side."""
        e = np.zeros(self.S + 2 * self.plane)
        if v is not None:
            e[self.plane:self.plane + self.S] = v
        return e


def _p(a, offset=0):
    return C.c_void_p(a.ctypes.data + offset * a.itemsize)


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    from oracle.oracle import Oracle
    lib = Oracle.lib()
    nx, ny, nz = LOCAL
    L, _, _, _ = Oracle.slab_hierarchy(nx, ny, nz, world)
    Oracle.colour_order(L)
    slabs = []
    for l, lev in enumerate(L):
        s = _Slab(lev, rank, nx >> l, ny >> l, nz >> l)
        if lev.f2c is not None:
            Sc = (nx >> (l + 1)) * (ny >> (l + 1)) * (nz >> (l + 1))
            s.f2c = np.ascontiguousarray(lev.f2c[rank * Sc:(rank + 1) * Sc] - rank * s.S)
            s.f2c = s.f2c.astype(np.int32)
        slabs.append(s)

    def exchange(s, e):
        """ExchangeHalo: own boundary planes out, the neighbours' into the halo."""
        reqs = []
        P, S = s.plane, s.S
        t = torch.from_numpy(e)
        if rank > 0:
            reqs.append(dist.isend(t[P:2 * P].clone(), rank - 1))
            lo = torch.empty(P, dtype=torch.float64)
            reqs.append(dist.irecv(lo, rank - 1))
        if rank + 1 < world:
            reqs.append(dist.isend(t[S:S + P].clone(), rank + 1))
            hi = torch.empty(P, dtype=torch.float64)
            reqs.append(dist.irecv(hi, rank + 1))
        for q in reqs:
            q.wait()
        if rank > 0:
            e[:P] = lo.numpy()
        if rank + 1 < world:
            e[S + P:] = hi.numpy()

    def symgs(s, r, e):
        exchange(s, e)
        lib.or_symgs(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(s.diag),
                     _p(s.order), _p(r), _p(e, s.plane))

    def spmv(s, e, y):
        exchange(s, e)
        lib.or_spmv(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(e, s.plane), _p(y))

    def mg(l, r, e):
        """ComputeMG_ref (src/ComputeMG_ref.cpp:39-63) on this rank."""
        s = slabs[l]
        e[:] = 0.0
        if s.f2c is None:
            symgs(s, r, e)
            return
        symgs(s, r, e)
        Axf = np.zeros(s.S)
        spmv(s, e, Axf)
        nc = s.f2c.size
        rc = np.zeros(nc)
        lib.or_restriction(C.c_int64(nc), _p(s.f2c), _p(r), _p(Axf), _p(rc))
        ec = slabs[l + 1].ext()
        mg(l + 1, rc, ec)
        xc = np.ascontiguousarray(ec[slabs[l + 1].plane:slabs[l + 1].plane + nc])
        xf = np.ascontiguousarray(e[s.plane:s.plane + s.S])
        lib.or_prolongation(C.c_int64(nc), _p(s.f2c), _p(xc), _p(xf))
        e[s.plane:s.plane + s.S] = xf
        symgs(s, r, e)

    def mg_fused(l, r, e, fix=True):
        """The library's order of the same V-cycle on a slab: the residual at
        the injected points is formed inside the pre-smoother with the halo
        the sweep read, then the halo is exchanged and only the first plane's
        injected residuals (the one plane that reads the halo below; the local
        z-extent is even) are formed again; the correction of the first plane
        is added before the exchange that precedes the post-smoother, the
        rest after it.  fix=False leaves the two fix-ups out (a planted
        mistake: the result must then differ)."""
        s = slabs[l]
        e[:] = 0.0                      # the first sweep's halo: zero, not exchanged
        lib.or_symgs(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(s.diag),
                     _p(s.order), _p(r), _p(e, s.plane))
        if s.f2c is None:
            return
        nc = s.f2c.size
        Axf = np.zeros(s.S)
        lib.or_spmv(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(e, s.plane), _p(Axf))
        rc = np.zeros(nc)
        lib.or_restriction(C.c_int64(nc), _p(s.f2c), _p(r), _p(Axf), _p(rc))
        exchange(s, e)
        first = s.f2c < s.plane          # injected points of the first plane
        assert (s.f2c[~first] >= s.plane).all()
        if rank > 0 and fix:
            lib.or_spmv(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(e, s.plane),
                        _p(Axf))
            rc[first] = r[s.f2c[first]] - Axf[s.f2c[first]]
        ec = slabs[l + 1].ext()
        mg_fused(l + 1, rc, ec, fix)
        xc = ec[slabs[l + 1].plane:slabs[l + 1].plane + nc]
        xf = e[s.plane:s.plane + s.S]
        if rank > 0 and fix:
            xf[s.f2c[first]] = xf[s.f2c[first]] + xc[first]
        exchange(s, e)
        rest = ~first if rank > 0 and fix else np.ones(nc, bool)
        xf[s.f2c[rest]] = xf[s.f2c[rest]] + xc[rest]
        lib.or_symgs(C.c_int64(s.S), _p(s.nnz), _p(s.cols), _p(s.vals), _p(s.diag),
                     _p(s.order), _p(r), _p(e, s.plane))

    def dot(x, y):
        """The ranks' partial dots added in rank order, as the oracle's
        restatement and the library's in-process group add them.  An
        all-reduce (MPI_Allreduce in src/ComputeDotProduct_ref.cpp:66-77,
        gloo's, NCCL's) fixes no order of the additions, which from three
        ranks on can change the last bits of the total."""
        local = torch.tensor([lib.or_dot(C.c_int64(x.size), _p(x), _p(y))], dtype=torch.float64)
        parts = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, local)
        total = 0.0
        for t in parts:
            total += float(t[0])
        return total

    def waxpby(a, x, b, y):
        w = np.zeros_like(x)
        lib.or_waxpby(C.c_int64(x.size), C.c_double(a), _p(x), C.c_double(b), _p(y), _p(w))
        return w

    s0 = slabs[0]
    n = L[0].nrow
    u = Oracle.uniform(11, n, 1.0, 2.0)
    rr = Oracle.uniform(12, n)
    x0 = Oracle.uniform(13, n)
    lo, hi = rank * s0.S, (rank + 1) * s0.S
    res = {}
    # one SYMGS from a non-zero start
    e = s0.ext(x0[lo:hi])
    symgs(s0, np.ascontiguousarray(rr[lo:hi]), e)
    res["symgs"] = e[s0.plane:s0.plane + s0.S].copy()
    # SpMV
    y = np.zeros(s0.S)
    spmv(s0, s0.ext(u[lo:hi]), y)
    res["spmv"] = y
    # V-cycle
    e = s0.ext()
    mg(0, np.ascontiguousarray(rr[lo:hi]), e)
    res["mg"] = e[s0.plane:s0.plane + s0.S].copy()
    e = s0.ext()
    mg_fused(0, np.ascontiguousarray(rr[lo:hi]), e)
    res["mg_fused"] = e[s0.plane:s0.plane + s0.S].copy()
    e = s0.ext()
    mg_fused(0, np.ascontiguousarray(rr[lo:hi]), e, fix=False)
    res["mg_nofix"] = e[s0.plane:s0.plane + s0.S].copy()
    # CG_ref (src/CG_ref.cpp:58-144), 12 iterations, with exchanges and all-reduces
    b = np.zeros(s0.S)
    spmv(s0, s0.ext(u[lo:hi]), b)
    x = np.zeros(s0.S)
    p = s0.ext(x)
    Ap = np.zeros(s0.S)
    spmv(s0, p, Ap)
    r_ = waxpby(1.0, b, -1.0, Ap)
    normr0 = normr = dot(r_, r_) ** 0.5
    rtz = 0.0
    for k in range(1, 13):
        ez = s0.ext()
        mg(0, r_, ez)
        z = np.ascontiguousarray(ez[s0.plane:s0.plane + s0.S])
        if k == 1:
            pv = z.copy()
            rtz = dot(r_, z)
        else:
            oldrtz, rtz = rtz, dot(r_, z)
            pv = waxpby(1.0, z, rtz / oldrtz, np.ascontiguousarray(p[s0.plane:s0.plane + s0.S]))
        p = s0.ext(pv)
        spmv(s0, p, Ap)
        alpha = rtz / dot(pv, Ap)
        x = waxpby(1.0, x, alpha, pv)
        r_ = waxpby(1.0, r_, -alpha, Ap)
        normr = dot(r_, r_) ** 0.5
    res["cg_x"] = x
    res["cg_normr"] = normr / normr0
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_oracle_matches_per_rank_exchange_gloo_ranks(world, oracle):
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    nx, ny, nz = LOCAL
    L, _, _, _ = oracle.slab_hierarchy(nx, ny, nz, world)
    oracle.colour_order(L)
    n = L[0].nrow
    u = oracle.uniform(11, n, 1.0, 2.0)
    rr = oracle.uniform(12, n)
    x0 = oracle.uniform(13, n)
    cat = lambda key: np.concatenate([out[r][key] for r in range(world)])  # noqa: E731
    assert (cat("spmv") == oracle.spmv(L[0], u)).all()
    assert (cat("symgs") == oracle.symgs(L[0], rr, x0, coloured=True)).all()
    assert (cat("mg") == oracle.mg(L, rr, coloured=True)).all()
    assert (cat("mg_fused") == cat("mg")).all()
    assert not (cat("mg_nofix") == cat("mg")).all()
    b = oracle.spmv(L[0], u)
    xs, k, nr, nr0 = oracle.cg(L, b, np.zeros(n), 12, 0.0, precond=True, coloured=True)
    assert k == 12
    assert (cat("cg_x") == xs).all()
    assert out[0]["cg_normr"] == nr / nr0


def test_slab_oracle_reduces_to_one_rank(oracle):
    """slab_rows = 0 (one rank) is the single-rank oracle; with two slabs the
    smoother differs (block Jacobi) but the SpMV does not."""
    L1, _, _, _ = oracle.hierarchy(16, 8, 16)
    L2, _, _, _ = oracle.slab_hierarchy(16, 8, 8, 2)
    for L in (L1, L2):
        oracle.colour_order(L)
    n = L1[0].nrow
    r, x0 = oracle.uniform(12, n), oracle.uniform(13, n)
    assert (oracle.spmv(L1[0], x0) == oracle.spmv(L2[0], x0)).all()
    g1 = oracle.symgs(L1[0], r, x0, coloured=True)
    g2 = oracle.symgs(L2[0], r, x0, coloured=True)
    assert not (g1 == g2).all()
    # from x = 0 the block-Jacobi sweep is a symmetric operator of r (one
    # symmetric Gauss-Seidel per slab), as the reference's preconditioner is
    M = np.stack([oracle.symgs(L2[0], np.eye(1, n, j)[0], np.zeros(n), coloured=True)
                  for j in range(6)])
    assert np.allclose(M[:, :6], M[:, :6].T, rtol=1e-12, atol=1e-15)
