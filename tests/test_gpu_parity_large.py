"""Parity at the benchmark grids: 256^3 (the plain FP64 configuration) against
the stored-matrix oracle, and 512^3 (the mixed-precision configuration, 134M
rows, 3.6e9 nonzeros) against the oracle's matrix-free restatements on every
row -- where storage-slot offsets pass 2^31, the grid reductions run over more
than 1024 blocks and the multiply-shift line mapping meets its largest
divisors.

Tolerances, as in test_gpu_parity.py: SpMV, SYMGS, MG, restriction,
prolongation, WAXPBY, residual and the mixed FP32/BF16 operators bit-exact
(``==``); dot products 1e-13 relative to the exactly rounded sum; CG after 10
iterations: same count,
initial norm 1e-14 and final norm 1e-8 relative.  SYMGS and MG are compared
with the reference's functions in colour order (the device sweeps colour by
colour).  The oracle's matrix-free functions are pinned to the stored-matrix
ones in tests/test_oracle_pin.py.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

D256 = (256, 256, 256)
D512 = (512, 512, 512)


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def g256(oracle):
    from hpcg_b200 import Problem
    L, b, _, _ = oracle.hierarchy(*D256)
    oracle.colour_order(L)
    P = Problem(*D256)
    P.generate("hpcg")            # the device generator, as the benchmark sets up
    n = L[0].nrow
    vecs = (oracle.uniform(11, n, 1.0, 2.0), oracle.uniform(12, n), oracle.uniform(13, n))
    yield L, b, P, vecs
    P.close()
    torch.cuda.empty_cache()


def test_256_generator_equals_host_load(g256):
    """The device-generated hierarchy holds exactly the values and columns of
    the reference hierarchy loaded from the host (OptimizeProblem's path)."""
    from hpcg_b200 import Problem
    L, _, P, _ = g256
    Q = Problem(*D256)
    try:
        for l, lev in enumerate(L):
            Q.load_level(l, lev.nnz, lev.cols, lev.vals)
            if lev.f2c is not None:
                Q.check_f2c(l, lev.f2c)
        for l in range(4):
            v1, c1 = P.get_values(l)
            v2, c2 = Q.get_values(l)
            assert torch.equal(v1, v2) and torch.equal(c1, c2)
            del v1, c1, v2, c2
    finally:
        Q.close()
        torch.cuda.empty_cache()


def test_256_spmv_both_column_forms(g256, oracle):
    L, _, P, (u, _, _) = g256
    for l, lev in enumerate(L):
        want = oracle.spmv(lev, u[:lev.nrow])
        x = cuda(u[:lev.nrow])
        assert (host(P.spmv(x, level=l)) == want).all()
        assert (host(P.spmv(x, level=l, stencil_cols=True)) == want).all()


def test_256_symgs_every_level(g256, oracle):
    L, _, P, (_, r, x0) = g256
    for l, lev in enumerate(L):
        n = lev.nrow
        x = cuda(x0[:n])
        P.symgs(cuda(r[:n]), x, level=l)
        assert (host(x) == oracle.symgs(lev, r[:n], x0[:n], coloured=True)).all()


def test_256_mg(g256, oracle):
    L, _, P, (_, r, _) = g256
    z = host(P.mg(cuda(r)))
    assert (z == oracle.mg(L, r, coloured=True)).all()


def test_256_restriction_prolongation(g256, oracle):
    L, _, P, (u, r, x0) = g256
    for l in range(3):
        n, nc = L[l].nrow, L[l + 1].nrow
        rc = host(P.restriction(l, cuda(r[:n]), cuda(u[:n])))
        assert (rc == oracle.restriction(L[l].f2c, r[:n], u[:n])).all()
        xf = host(P.prolongation(l, cuda(u[:nc]), cuda(x0[:n])))
        assert (xf == oracle.prolongation(L[l].f2c, u[:nc], x0[:n])).all()


def test_256_vector_ops(g256, oracle):
    """Dot products: 1e-13 relative to the exactly rounded sum of the same
    (rounded) products, math.fsum.  The oracle's left-to-right sum of 16.8M
    terms itself drifts by about 1e-13 from it (measured: 1.3e-13 for u.u), and
    the reference's OpenMP reduction order is a third order, so the oracle is
    held to 1e-12 of the exact sum and the device to 1e-13."""
    import math
    _, _, P, (u, r, _) = g256
    du, dr = cuda(u), cuda(r)
    for a, b, da, db in ((u, r, du, dr), (u, u, du, du)):
        exact = math.fsum(a * b)
        assert abs(P.dot(da, db) / exact - 1) < 1e-13
        assert abs(oracle.dot(a, b) / exact - 1) < 1e-12
    for a, bb in ((1.0, 0.37), (-0.61, 1.0), (0.83, -1.29)):
        assert (host(P.waxpby(a, du, bb, dr)) == oracle.waxpby(a, u, bb, r)).all()
    assert P.residual(du, dr) == oracle.residual(u, r)


def test_256_mixed_operators(g256, oracle):
    L, _, P, (u, r, x0) = g256
    P.build_mixed()
    for l, lev in enumerate(L):
        n = lev.nrow
        u32 = u[:n].astype(np.float32)
        assert (host(P.spmv_mixed(cuda(u32), level=l)) == oracle.spmv32(lev, u32)).all()
        x32 = x0[:n].astype(np.float32)
        rr = r[:n] if l == 0 else r[:n].astype(np.float32)
        xd = cuda(x32)
        P.symgs_mixed(cuda(rr), xd, level=l)
        assert (host(xd) == oracle.symgs32(lev, rr, x32)).all()
    assert (host(P.mg_mixed(cuda(r))) == oracle.mg32(L, r)).all()


def test_256_cg_10_iterations(g256, oracle):
    """CG_ref's 10 iterations on the colour-permuted matrix (src/CG_ref.cpp:58-144)."""
    L, b, P, _ = g256
    n = L[0].nrow
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    k, nr, nr0 = P.cg(cuda(b), x, 10, 0.0)
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 10, 0.0, coloured=True)
    assert k == ok == 10
    assert abs(nr0 / onr0 - 1) < 1e-14 and abs(nr / onr - 1) < 1e-8
    assert np.abs(host(x) - ox).max() < 1e-10


def test_512_every_row(oracle):
    """512^3, device-generated as the benchmark does: SpMV in both column forms,
    the finest-level FP64 symmetric sweep and the finest-level mixed sweep,
    each on all 134,217,728 rows against the matrix-free oracle; A*1 = b
    exactly (src/GenerateProblem_ref.cpp:178-180)."""
    from hpcg_b200 import Problem
    torch.cuda.empty_cache()
    P = Problem(*D512)
    try:
        P.generate("hpcg")
        n = P.rows()
        u = oracle.uniform(21, n, -1.0, 1.0)
        want = oracle.stencil_spmv(D512, u)
        du = cuda(u)
        assert (host(P.spmv(du, level=0)) == want).all()
        assert (host(P.spmv(du, level=0, stencil_cols=True)) == want).all()
        ones = np.ones(n)
        b = oracle.stencil_spmv(D512, ones)
        assert P.residual(P.spmv(cuda(ones)), cuda(b)) == 0.0
        del du
        r = oracle.uniform(22, n)
        x0 = oracle.uniform(23, n, 1.0, 2.0)
        x = cuda(x0)
        P.symgs(cuda(r), x, level=0)
        assert (host(x) == oracle.stencil_symgs(D512, r, x0)).all()
        del x
        P.build_mixed()
        x32 = x0.astype(np.float32)
        xd = cuda(x32)
        P.symgs_mixed(cuda(r), xd, level=0)
        assert (host(xd) == oracle.stencil_symgs32(D512, r, x32)).all()
    finally:
        P.close()
        torch.cuda.empty_cache()
