"""The Python host API's argument checks, on the CPU with a stand-in library.

The C ABI takes raw pointers and cannot tell a host array, a tensor of another
device, a strided view or a short vector from a good device vector; the GPU
would dereference any of them.  ``Problem`` and ``Group`` check every vector
before the call: these tests run each operator against a fake library that
records its calls, with CPU tensors standing for the problem's device, and
check that good arguments reach the library as the tensors' own pointers and
that bad ones are refused before any library call."""
import ctypes as C

import numpy as np
import pytest
import torch

GRID = (8, 8, 8)


class FakeLib:
    """Records hpcgx_* calls; hpcgx_rows answers from the grid."""

    def __init__(self, dims=GRID, levels=4):
        self.dims, self.levels, self.calls = dims, levels, []

    def hpcgx_rows(self, h, level):
        if not 0 <= level < self.levels:
            return -1
        nx, ny, nz = self.dims
        return (nx >> level) * (ny >> level) * (nz >> level)

    def __getattr__(self, name):
        if not name.startswith("hpcgx_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append((name, args))
            return 0
        return call


@pytest.fixture
def api(monkeypatch):
    from hpcg_b200 import problem as pm
    fake = FakeLib()
    monkeypatch.setattr(pm, "lib", lambda: fake)
    monkeypatch.setattr(pm.Problem, "_pre", lambda self: None)

    made = []

    def make(dims=GRID, rank=0, nranks=1):
        P = pm.Problem.__new__(pm.Problem)
        P.dims, P.levels, P.nranks, P.rank = dims, 4, nranks, rank
        P.device = torch.device("cpu")
        P.h = C.c_void_p(1)          # a dummy handle: only the fake library sees it
        P.values_version = 0
        made.append(P)
        return P
    yield pm, fake, make
    for P in made:                   # never hand the dummy handle to the real library
        P.h = None


def ptr(a):
    v = a.value if isinstance(a, C.c_void_p) else a
    return v


def test_good_arguments_reach_the_library_unchanged(api):
    pm, fake, make = api
    P = make()
    n = P.rows(0)
    x, r = torch.rand(n, dtype=torch.float64), torch.rand(n, dtype=torch.float64)
    y = P.spmv(x)
    name, args = fake.calls[-1]
    assert name == "hpcgx_spmv" and ptr(args[2]) == x.data_ptr() and ptr(args[3]) == y.data_ptr()
    P.spmv(x, y=y, stencil_cols=True)
    assert fake.calls[-1][0] == "hpcgx_spmv_stencil"
    P.symgs(r, x, level=0)
    assert [ptr(a) for a in fake.calls[-1][1][2:]] == [r.data_ptr(), x.data_ptr()]
    P.mg(r)
    n1 = P.rows(1)
    P.restriction(0, r, x)
    P.prolongation(0, torch.zeros(n1, dtype=torch.float64), x)
    # vector operations take n from x; longer y / w are fine
    assert P.dot(x, r) == 0.0 and fake.calls[-1][1][1] == n
    P.dot(x[:10], r)
    assert fake.calls[-1][1][1] == 10
    w = P.waxpby(1.0, x, 0.5, r)
    assert ptr(fake.calls[-1][1][6]) == w.data_ptr()
    P.waxpby(1.0, x, 0.5, r, w=x)          # aliasing w == x, as CG uses it
    P.residual(x, r)
    x32 = torch.zeros(n, dtype=torch.float32)
    P.spmv_mixed(x32)
    for rr in (r, r.float()):               # FP64 or FP32 right-hand side
        P.symgs_mixed(rr, x32)
        _, args = fake.calls[-1]
        assert (args[2] is None) == (rr.dtype == torch.float32)
        assert (args[3] is None) == (rr.dtype == torch.float64)
    P.mg_mixed(r)
    P.cg(r, x, 10, 0.0)
    P.cg_mixed(r, x, 10, 0.0, times=np.zeros(10))
    P.cg_host(r.numpy(), x.numpy().copy(), 10, 0.0)
    P.cg_host(r, x, 10, 0.0, mixed=True)    # CPU tensors are host memory here
    P.adjoint_grad(r, x)
    P.set_values(torch.zeros(27 * n, dtype=torch.float64))
    assert [c[0] for c in fake.calls].count("hpcgx_cg_host") == 2


BAD = [
    ("float32 where float64", lambda n: torch.zeros(n, dtype=torch.float32), TypeError),
    ("short", lambda n: torch.zeros(n - 1, dtype=torch.float64), ValueError),
    ("strided", lambda n: torch.zeros(2 * n, dtype=torch.float64)[::2], ValueError),
    ("host array", lambda n: np.zeros(n), TypeError),
    ("other device", lambda n: torch.empty(n, dtype=torch.float64, device="meta"), ValueError),
]


@pytest.mark.parametrize("what,make_bad,exc", BAD, ids=[b[0] for b in BAD])
def test_bad_vectors_are_refused_before_any_call(api, what, make_bad, exc):
    pm, fake, make = api
    P = make()
    n = P.rows(0)
    good = torch.zeros(n, dtype=torch.float64)
    bad = make_bad(n)
    calls = [
        lambda: P.spmv(bad), lambda: P.spmv(good, y=bad), lambda: P.symgs(bad, good),
        lambda: P.symgs(good, bad), lambda: P.mg(bad), lambda: P.mg(good, bad),
        lambda: P.restriction(0, bad, good), lambda: P.prolongation(0, good[:P.rows(1)], bad),
        lambda: P.cg(bad, good, 1, 0.0), lambda: P.cg(good, bad, 1, 0.0),
        lambda: P.cg_mixed(good, bad, 1, 0.0), lambda: P.mg_mixed(bad),
        lambda: P.adjoint_grad(bad, good), lambda: P.dot(good, bad),
        lambda: P.waxpby(1.0, good, 1.0, bad), lambda: P.waxpby(1.0, good, 1.0, good, w=bad),
        lambda: P.residual(good, bad),
    ]
    for i, f in enumerate(calls):
        with pytest.raises(exc):
            f()
        assert fake.calls == [], i


def test_mixed_and_host_arguments_checked(api):
    pm, fake, make = api
    P = make()
    n = P.rows(0)
    x64 = torch.zeros(n, dtype=torch.float64)
    with pytest.raises(TypeError):
        P.spmv_mixed(x64)                                  # FP32 vector expected
    with pytest.raises(TypeError):
        P.symgs_mixed(torch.zeros(n, dtype=torch.float16), torch.zeros(n))
    with pytest.raises(TypeError):
        P.symgs_mixed(x64, x64)                            # x is FP32
    with pytest.raises(TypeError):
        P.cg_host(np.zeros(n, np.float32), np.zeros(n), 1, 0.0)
    with pytest.raises(ValueError):
        P.cg_host(np.zeros(n), np.zeros(n - 1), 1, 0.0)
    with pytest.raises(ValueError):
        P.cg_host(np.zeros(n), np.zeros((n, 2))[:, 0], 1, 0.0)   # strided output
    with pytest.raises(ValueError):
        P.cg(x64, x64.clone(), 1, 0.0, times=np.zeros(3))       # CG adds to times[5]
    with pytest.raises(ValueError):
        P.set_values(torch.zeros(27 * n - 1, dtype=torch.float64))
    assert fake.calls == []


def test_host_matrix_loads_checked(api):
    pm, fake, make = api
    P = make()
    n = P.rows(0)
    nnz, cols, vals = np.full(n, 27, np.uint8), np.zeros(27 * n, np.int32), np.zeros(27 * n)
    P.load_level(0, nnz, cols, vals)
    assert fake.calls[-1][0] == "hpcgx_load_level"
    for args in ((nnz[:-1], cols, vals), (nnz, cols[:-1], vals), (nnz, cols, vals[:-27])):
        with pytest.raises(ValueError):
            P.load_level(0, *args)
    with pytest.raises(ValueError):
        P.set_diagonal(0, np.zeros(n - 1))
    # a row wider than 27 still reaches the library, which names the row
    wide = nnz.copy()
    wide[5] = 28
    P.load_level(0, wide, cols, vals)
    assert fake.calls[-1][0] == "hpcgx_load_level"


def test_general_rows_checked(api):
    pm, fake, make = api
    P = make()
    P.dims = None
    m, w = 6, 4
    nnz = np.array([1, 2, 3, 4, 2, 1], np.uint8)
    cols = np.zeros((m, w), np.int32)
    vals = np.zeros((m, w))
    P.load_level_general(0, nnz, cols, vals)
    name, args = fake.calls[-1]
    assert name == "hpcgx_load_level_general" and args[2] == m
    # row pointers step by the arrays' width
    assert [args[4][i] - args[4][0] for i in range(m)] == [4 * w * i for i in range(m)]
    assert [args[5][i] - args[5][0] for i in range(m)] == [8 * w * i for i in range(m)]
    fake.calls.clear()
    wide = nnz.copy()
    wide[2] = w + 1                                   # would read into the next row
    for a in ((wide, cols, vals), (nnz[:-1], cols, vals), (nnz, cols, vals[:, :3]),
              (nnz, cols.reshape(-1), vals.reshape(-1))):
        with pytest.raises(ValueError):
            P.load_level_general(0, *a)
    assert fake.calls == []


def test_group_vector_lists_checked(api):
    pm, fake, make = api
    ranks = [make(rank=r, nranks=2) for r in range(2)]
    g = pm.Group.__new__(pm.Group)
    g.ranks, g.g, g.stream = ranks, C.c_void_p(2), None
    monkey_pre = pm.Group._pre
    pm.Group._pre = lambda self: None
    try:
        n = ranks[0].rows(0)
        xs = [torch.rand(n, dtype=torch.float64) for _ in ranks]
        ys = g.spmv(xs)
        name, args = fake.calls[-1]
        assert name == "hpcgx_group_spmv"
        assert [args[2][i] for i in range(2)] == [x.data_ptr() for x in xs]
        assert [args[3][i] for i in range(2)] == [y.data_ptr() for y in ys]
        g.symgs([x[:ranks[0].rows(1)].contiguous() for x in xs],
                [torch.zeros(ranks[0].rows(1), dtype=torch.float64) for _ in ranks], level=1)
        g.mg(xs)
        g.cg(xs, [torch.zeros(n, dtype=torch.float64) for _ in ranks], 5, 0.0)
        fake.calls.clear()
        with pytest.raises(ValueError):
            g.spmv(xs[:1])                                 # one vector per rank
        with pytest.raises(ValueError):
            g.mg([xs[0], xs[1][:-1]])
        with pytest.raises(TypeError):
            g.cg(xs, [torch.zeros(n, dtype=torch.float32) for _ in ranks], 5, 0.0)
        assert fake.calls == []
    finally:
        pm.Group._pre = monkey_pre
        g.g = None
