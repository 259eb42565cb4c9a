"""General-pattern problems (hpcgx_create_general) against the oracle.

The reference requires that an implementation work for general unstructured
sparse matrices (src/GenerateProblem.cpp:47-49).  Two kinds of input that the
stencil layout cannot take:

* HPCG's hierarchy under a random symmetric renumbering of every level
  (rows, columns and the injection f2c renumbered alike): the same operator
  with no grid structure left in its natural order;
* a random sparse SPD matrix (a weighted graph Laplacian plus the identity)
  with rows of 2 to 27 entries.

Oracle: the reference's functions restated in oracle/hpcg_oracle.c on the same
host matrices -- ComputeSPMV_ref, ComputeSYMGS_ref on the matrix permuted by the
greedy multicolouring of src/OptimizeProblem.cpp:50-79 (or_greedy_colour),
ComputeMG_ref and CG_ref.  Tolerances as for the stencil path: SpMV, SYMGS and
MG bit-exact; CG the same iteration count to 1e-10 and residual norms within
1e-8 relative after 10 iterations.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def renumbered_hierarchy(oracle, dims, seed):
    """HPCG's hierarchy with every level's rows renumbered by a random
    permutation (new index = perm[old]); each row keeps its entry order."""
    from oracle.oracle import Level
    L, b, _, _ = oracle.hierarchy(*dims)
    rng = np.random.default_rng(seed)
    perms = [rng.permutation(lev.nrow).astype(np.int64) for lev in L]
    out = []
    for l, lev in enumerate(L):
        p = perms[l]
        n = lev.nrow
        inv = np.empty(n, np.int64)
        inv[p] = np.arange(n)
        cols = lev.cols.reshape(n, 27)[inv]
        vals = lev.vals.reshape(n, 27)[inv].copy()
        nnz = lev.nnz[inv].copy()
        mask = np.arange(27)[None, :] < nnz[:, None]
        cols = np.where(mask, p[cols], np.arange(n)[:, None]).astype(np.int32)
        diag = lev.diag[inv].copy()
        f2c = None
        if lev.f2c is not None:
            pc = perms[l + 1]
            invc = np.empty(pc.size, np.int64)
            invc[pc] = np.arange(pc.size)
            f2c = p[lev.f2c[invc]].astype(np.int32)
        new = Level(lev.nx, lev.ny, lev.nz, np.ascontiguousarray(nnz),
                    np.ascontiguousarray(cols.reshape(-1)), np.ascontiguousarray(vals.reshape(-1)),
                    np.ascontiguousarray(diag), f2c)
        out.append(new)
    return out, p_vec(b, perms[0])


def p_vec(v, p):
    w = np.empty_like(v)
    w[p] = v
    return w


def random_spd(oracle, n, seed):
    """Weighted graph Laplacian + I on a random graph, rows of 2..27 entries,
    entries in increasing column order (one level)."""
    from oracle.oracle import Level
    rng = np.random.default_rng(seed)
    nb = [set() for _ in range(n)]
    for i in range(n):
        for j in rng.choice(n, size=rng.integers(1, 10), replace=False):
            if j != i and len(nb[i]) < 26 and len(nb[j]) < 26:
                nb[i].add(int(j))
                nb[j].add(i)
    w = {}
    cols = np.zeros((n, 27), np.int32)
    vals = np.zeros((n, 27))
    nnz = np.zeros(n, np.uint8)
    diag = np.zeros(n, np.int32)
    for i in range(n):
        row = sorted(nb[i] | {i})
        nnz[i] = len(row)
        d = 1.0
        for k, j in enumerate(row):
            cols[i, k] = j
            if j != i:
                key = (min(i, j), max(i, j))
                if key not in w:
                    w[key] = float(rng.uniform(0.5, 2.0))
                vals[i, k] = -w[key]
                d += w[key]
            else:
                diag[i] = k
        vals[i, diag[i]] = d
        cols[i, nnz[i]:] = i
    lev = Level(n, 1, 1, nnz, cols.reshape(-1), vals.reshape(-1), diag, None)
    return [lev]


def load(P, L):
    for l, lev in enumerate(L):
        P.load_level_general(l, lev.nnz, lev.cols.reshape(lev.nrow, 27),
                             lev.vals.reshape(lev.nrow, 27), lev.f2c)


CASES = [("renumbered16", (16, 16, 16)), ("renumbered24x16x8", (24, 16, 8)), ("random", 6000)]


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def case(request, oracle):
    from hpcg_b200 import Problem
    name, arg = request.param
    if name == "random":
        L = random_spd(oracle, arg, 7)
        b = oracle.spmv(L[0], oracle.uniform(5, L[0].nrow, -1.0, 1.0))
    else:
        L, b = renumbered_hierarchy(oracle, arg, 3)
    oracle.colour_order(L)
    P = Problem.general(levels=len(L))
    load(P, L)
    yield L, b, P
    P.close()


def test_colouring_from_the_graph(case):
    L, b, P = case
    for l, lev in enumerate(L):
        assert P.colours(l) == lev.ncolors
        # a proper colouring: no entry joins two rows of one colour
        n = lev.nrow
        rows = np.repeat(np.arange(n), 27)
        ok = np.arange(27 * n) % 27 < np.repeat(lev.nnz, 27)
        r, c = rows[ok], lev.cols[ok]
        off = r != c
        assert (lev.colors[r[off]] != lev.colors[c[off]]).all()


def test_general_spmv_symgs_mg_bitexact(case, oracle):
    L, b, P = case
    n = L[0].nrow
    u, r, x0 = oracle.uniform(11, n, 1.0, 2.0), oracle.uniform(12, n), oracle.uniform(13, n)
    for l, lev in enumerate(L):
        m = lev.nrow
        assert (host(P.spmv(cuda(u[:m]), level=l)) == oracle.spmv(lev, u[:m])).all()
        x = cuda(x0[:m])
        P.symgs(cuda(r[:m]), x, level=l)
        assert (host(x) == oracle.symgs(lev, r[:m], x0[:m], coloured=True)).all()
    z = host(P.mg(cuda(r)))
    assert (z == oracle.mg(L, r, coloured=True)).all()
    # host-buffer forms (the drop-in's path) agree with the device forms
    xh = x0.copy()
    from hpcg_b200._lib import lib
    import ctypes as C
    assert lib().hpcgx_symgs_host(P.h, 0, r.ctypes.data_as(C.c_void_p),
                                  xh.ctypes.data_as(C.c_void_p)) == 0
    assert (xh == oracle.symgs(L[0], r, x0, coloured=True)).all()


def test_general_cg(case, oracle):
    L, b, P = case
    n = L[0].nrow
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    k, nr, nr0 = P.cg(cuda(b), x, 10, 0.0)
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 10, 0.0, coloured=True)
    assert k == ok == 10 and abs(nr0 / onr0 - 1) < 1e-14 and abs(nr / onr - 1) < 1e-8
    x.zero_()
    k, nr, nr0 = P.cg(cuda(b), x, 1000, 1e-10)
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 1000, 1e-10, coloured=True)
    assert k == ok and nr / nr0 <= 1e-10
    x.zero_()
    k, nr, nr0 = P.cg(cuda(b), x, 30, 0.0, precond=False)
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 30, 0.0, precond=False)
    assert k == ok and abs(nr / onr - 1) < 1e-6


def test_general_diagonal_and_refusals(oracle):
    from hpcg_b200 import HPCGXError, Problem
    L = random_spd(oracle, 500, 9)
    P = Problem.general(levels=1)
    lev = L[0]
    # a row without its diagonal entry, a column out of range: HPCGX_ELAYOUT
    vals = lev.vals.reshape(500, 27)
    cols = lev.cols.reshape(500, 27).copy()
    i = int(np.argmax(lev.nnz >= 2))
    j = int(lev.diag[i])
    cols[i, j] = cols[i, 1 if j == 0 else 0]          # the row loses its diagonal entry
    with pytest.raises(HPCGXError) as e:
        P.load_level_general(0, lev.nnz, cols, vals)
    assert e.value.code == 5
    cols2 = lev.cols.reshape(500, 27).copy()
    cols2[7, 0] = 10**6
    with pytest.raises(HPCGXError) as e:
        P.load_level_general(0, lev.nnz, cols2, vals)
    assert e.value.code == 5
    load(P, L)
    d = P.get_diagonal(0)
    assert (d == vals[np.arange(500), lev.diag]).all()
    P.set_diagonal(0, d * 2.0)
    assert (P.get_diagonal(0) == d * 2.0).all()
    P.set_diagonal(0, d)
    # stencil-only entry points refuse a general problem
    b = torch.ones(500, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    with pytest.raises(HPCGXError) as e:
        P.cg_mixed(b, x, 10, 0.0)
    assert e.value.code == 3
    with pytest.raises(HPCGXError) as e:
        P.generate("hpcg")
    assert e.value.code == 3
    P.close()
