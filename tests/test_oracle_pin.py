"""Pins the oracle (oracle/hpcg_oracle.c) before anything is checked against it.

1. Against the golden vectors in tests/golden/, which are outputs of the
   reference's own code (tests/golden/make_golden.py): bit-exact for SpMV,
   SYMGS, MG, restriction, prolongation, WAXPBY and the residual norm; dot
   products to 1e-13 relative (the reference's OpenMP reduction order differs
   from a sequential sum).
2. Against the reference's structural checks (CheckProblem) and known answers:
   A * xexact == b exactly; greedy colouring yields 8 colours.
3. Live against oracle/_ref (the reference compiled from its sources) when it
   is present, on inputs the fixtures do not hold.
"""
import numpy as np
import pytest

from conftest import GOLDEN_GRIDS, load_golden


@pytest.fixture(scope="module", params=GOLDEN_GRIDS, ids=lambda d: "x".join(map(str, d)))
def case(request, oracle):
    dims = request.param
    L, b, x, xe = oracle.hierarchy(*dims)
    oracle.colour_order(L)
    return dims, L, b, xe, load_golden(dims)


def inputs(oracle, n):
    return oracle.uniform(11, n, 1.0, 2.0), oracle.uniform(12, n), oracle.uniform(13, n)


def test_check_problem_all_levels(case, oracle):
    from oracle.oracle import Oracle, _ptr
    dims, L, b, xe, g = case
    for l, lev in enumerate(L):
        args = [_ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals), _ptr(lev.diag)]
        vecs = [_ptr(b), _ptr(np.zeros(lev.nrow)), _ptr(xe)] if l == 0 else [None, None, None]
        assert Oracle.lib().or_check_problem(lev.nx, lev.ny, lev.nz, *args, *vecs) == 0
    assert (b == g["b"]).all()


def test_exact_solution_known_answer(case, oracle):
    dims, L, b, xe, g = case
    assert oracle.residual(oracle.spmv(L[0], xe), b) == 0.0
    assert g["A_xexact_resid"][0] == 0.0


def test_greedy_colouring_is_parity_8_colours(case):
    from oracle.oracle import geometric_colour
    dims, L, b, xe, g = case
    for lev in L:
        assert lev.ncolors == 8
        assert (lev.colors == geometric_colour(lev.nx, lev.ny, lev.nz)).all()


def test_colours_are_independent_sets(case):
    """No two rows of one colour share a stencil edge, on every level: the rows
    of a colour may be updated in any order (in parallel)."""
    dims, L, b, xe, g = case
    for lev in L:
        rows = np.repeat(np.arange(lev.nrow), 27)
        used = (np.arange(27)[None, :] < lev.nnz[:, None].astype(np.int64)).ravel()
        i, j = rows[used], lev.cols.astype(np.int64)[used]
        off = i != j
        assert (lev.colors[i[off]] != lev.colors[j[off]]).all()


def test_spmv_and_symgs_bitexact(case, oracle):
    dims, L, b, xe, g = case
    u, r, x0 = inputs(oracle, L[0].nrow)
    for l, lev in enumerate(L):
        n = lev.nrow
        assert (oracle.spmv(lev, u[:n]) == g["spmv_L%d" % l]).all()
        assert (oracle.symgs(lev, r[:n], x0[:n], coloured=True) == g["symgs_perm_L%d" % l]).all()
    assert (oracle.symgs(L[0], r, x0) == g["symgs_L0"]).all()


def test_mg_bitexact(case, oracle):
    dims, L, b, xe, g = case
    u, r, x0 = inputs(oracle, L[0].nrow)
    assert (oracle.mg(L, r) == g["mg"]).all()
    assert (oracle.mg(L, r, coloured=True) == g["mg_perm"]).all()


def test_transfer_and_vector_ops(case, oracle):
    dims, L, b, xe, g = case
    u, r, x0 = inputs(oracle, L[0].nrow)
    nc = L[1].nrow
    assert (oracle.restriction(L[0].f2c, r, u) == g["restriction_L0"]).all()
    assert (oracle.prolongation(L[0].f2c, u[:nc], x0) == g["prolongation_L0"]).all()
    assert (oracle.waxpby(1.0, u, 0.37, r) == g["waxpby_a1"]).all()
    assert (oracle.waxpby(-0.61, u, 1.0, r) == g["waxpby_b1"]).all()
    assert (oracle.waxpby(0.83, u, -1.29, r) == g["waxpby_ab"]).all()
    assert oracle.residual(u, r) == g["residual_ur"][0]
    assert abs(oracle.dot(u, r) / g["dot_ur"][0] - 1) < 1e-13
    assert abs(oracle.dot(u, u) / g["dot_uu"][0] - 1) < 1e-13


def test_cg_trajectory(case, oracle):
    dims, L, b, xe, g = case
    n = L[0].nrow
    for coloured, tag in ((False, "cg10"), (True, "cg10_perm")):
        x, k, nr, nr0 = oracle.cg(L, b, np.zeros(n), 10, 0.0, coloured=coloured)
        kk, gnr, gnr0 = g[tag + "_stats"]
        assert k == kk and abs(nr0 / gnr0 - 1) < 1e-14
        assert abs(nr / gnr - 1) < 1e-8
        assert np.abs(x - g[tag + "_x"]).max() < 1e-10
    for coloured, tag in ((False, "cgtol"), (True, "cgtol_perm")):
        x, k, nr, nr0 = oracle.cg(L, b, np.zeros(n), 500, 1e-10, coloured=coloured)
        assert k == g[tag + "_stats"][0]


def test_testcg_iteration_counts(case, oracle):
    """TestCG (src/TestCG.cpp:62-111) on the oracle: <= 12 / <= 2 iterations."""
    dims, L, b, xe, g = case
    n = L[0].nrow
    scale = np.full(n, 1.0e6)
    scale[:9] = (np.arange(9) + 2) * 1.0e6
    lev = L[0]
    saved = lev.vals.copy()
    idx = np.arange(n) * 27 + lev.diag
    lev.vals[idx] *= scale
    try:
        for prec, tag, limit in ((False, "testcg_noprec", 12), (True, "testcg_prec", 2)):
            _, k, nr, nr0 = oracle.cg(L, b * scale, np.zeros(n), 50, 1e-12, precond=prec)
            assert k == g[tag][0] and k <= limit
    finally:
        lev.vals[:] = saved


@pytest.mark.parametrize("dims", [(24, 16, 32), (40, 24, 56), (64, 32, 16)],
                         ids=lambda d: "x".join(map(str, d)))
def test_live_against_reference_build(dims, oracle):
    """Fresh seeds against the reference compiled from its sources, on the
    GPU tests' non-cubic grids too (odd coarsest levels: 5 x 3 x 7)."""
    from oracle.oracle import RefProblem
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    ref = RefProblem(*dims)
    L, b, _, _ = oracle.hierarchy(*dims)
    oracle.colour_order(L)
    ref.build_permuted([lev.position for lev in L])
    n = L[0].nrow
    u, r, x0 = oracle.uniform(101, n, -1, 1), oracle.uniform(102, n), oracle.uniform(103, n)
    for l, lev in enumerate(L):
        m = lev.nrow
        assert (oracle.spmv(lev, u[:m]) == ref.spmv(l, u[:m])).all()
        assert (oracle.symgs(lev, r[:m], x0[:m]) == ref.symgs(l, r[:m], x0[:m])).all()
        assert (oracle.symgs(lev, r[:m], x0[:m], coloured=True) ==
                ref.symgs_permuted(l, r[:m], x0[:m])).all()
    assert (oracle.mg(L, r) == ref.mg(r)).all()
    assert (oracle.mg(L, r, coloured=True) == ref.mg_permuted(r)).all()
    # CG_ref's trajectory (src/CG_ref.cpp:58-144), natural and colour order:
    # same iteration count, norms within 1e-8 after 10 iterations (the
    # reference's dot products sum in OpenMP's order)
    b = oracle.spmv(L[0], u)
    for coloured in (False, True):
        f = ref.cg_permuted if coloured else ref.cg
        got = f(b, np.zeros(n), 10, 0.0)
        ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 10, 0.0, coloured=coloured)
        assert got[1] == ok == 10
        assert abs(got[3] / onr0 - 1) < 1e-13 and abs(got[2] / onr - 1) < 1e-8
        assert np.abs(got[0] - ox).max() < 1e-10 * np.abs(ox).max()
    ref.close()


ODD_GRIDS = [(15, 13, 11, 1), (9, 7, 5, 1), (1, 6, 3, 1), (3, 1, 2, 1), (1, 1, 1, 1),
             (65, 13, 11, 1), (30, 26, 22, 2), (40, 24, 56, 3), (128, 40, 24, 2)]


@pytest.mark.parametrize("grid", ODD_GRIDS, ids=lambda d: "x".join(map(str, d[:3])) + f"_l{d[3]}")
def test_live_reference_on_odd_and_shallow_grids(grid, oracle):
    """The grids of the GPU's odd-grid tests, against the reference built
    with as many levels as the grid coarsens (odd, degenerate and single-row
    grids; 1 to 3 levels): the generated matrix and injection, SpMV, SYMGS in
    natural and colour order, the V-cycle and CG_ref's trajectory."""
    from oracle.oracle import RefProblem
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    nx, ny, nz, levels = grid
    ref = RefProblem(nx, ny, nz, levels=levels)
    try:
        L, b, _, _ = oracle.hierarchy(nx, ny, nz, levels=levels)
        oracle.colour_order(L)
        ref.build_permuted([lev.position for lev in L])
        for l, lev in enumerate(L):
            got = ref.export_level(l)
            assert (got.nnz == lev.nnz).all() and (got.cols == lev.cols).all()
            assert (got.vals == lev.vals).all() and (got.diag == lev.diag).all()
            assert (got.f2c is None) == (lev.f2c is None)
            if lev.f2c is not None:
                assert (got.f2c == lev.f2c).all()
        n = L[0].nrow
        u, r, x0 = oracle.uniform(111, n, -1, 1), oracle.uniform(112, n), oracle.uniform(113, n)
        for l, lev in enumerate(L):
            m = lev.nrow
            assert (oracle.spmv(lev, u[:m]) == ref.spmv(l, u[:m])).all()
            assert (oracle.symgs(lev, r[:m], x0[:m]) == ref.symgs(l, r[:m], x0[:m])).all()
            assert (oracle.symgs(lev, r[:m], x0[:m], coloured=True) ==
                    ref.symgs_permuted(l, r[:m], x0[:m])).all()
        assert (oracle.mg(L, r) == ref.mg(r)).all()
        assert (oracle.mg(L, r, coloured=True) == ref.mg_permuted(r)).all()
        bb = oracle.spmv(L[0], u)
        for coloured in (False, True):
            f = ref.cg_permuted if coloured else ref.cg
            got = f(bb, np.zeros(n), 10, 0.0)
            ox, ok, onr, onr0 = oracle.cg(L, bb, np.zeros(n), 10, 0.0, coloured=coloured)
            assert got[1] == ok
            assert abs(got[3] / onr0 - 1) < 1e-13
            # within 1e-8 of each other, or both at the round-off floor
            assert abs(got[2] - onr) <= 1e-8 * onr + 1e-13 * onr0
            assert np.abs(got[0] - ox).max() <= 1e-10 * np.abs(ox).max()
    finally:
        ref.close()


def test_mixed_oracle_consistency(oracle):
    """The FP32/BF16 restatement reduces to exact BF16 values on the HPCG
    stencil (26 and -1 are BF16-exact) and its flexible CG converges."""
    dims = (16, 16, 16)
    L, b, _, _ = oracle.hierarchy(*dims)
    oracle.colour_order(L)
    for lev in L:
        v16 = lev.vals_bf16.astype(np.uint32) << 16
        assert (v16.view(np.float32).astype(np.float64) == lev.vals).all()
    x, k, nr, nr0 = oracle.fcg(L, b, np.zeros(L[0].nrow), 200, 1e-10)
    assert nr / nr0 <= 1e-10 and k < 40


def test_varcoef_generator_properties(oracle):
    """Symmetric, diagonal = sum|offdiag| + 2, coarse levels follow the
    finest field at the injected points."""
    L, _, _, _ = oracle.hierarchy(16, 16, 16, varcoef=(2, 0.5))
    for lev in L:
        n = lev.nrow
        A = {}
        for i in range(n):
            for j in range(lev.nnz[i]):
                A[(i, int(lev.cols[i * 27 + j]))] = lev.vals[i * 27 + j]
        for (i, j), v in A.items():
            assert A[(j, i)] == v
        for i in range(n):
            off = sum(abs(A[(i, int(lev.cols[i * 27 + j]))]) for j in range(lev.nnz[i])
                      if lev.cols[i * 27 + j] != i)
            assert abs(A[(i, i)] - (off + 2.0)) <= 1e-12 * A[(i, i)]


def test_varcoef_cg_against_reference(oracle):
    """CG_ref of the reference build on the variable-coefficient hierarchy
    agrees with the oracle's CG (both natural order)."""
    from oracle.oracle import RefProblem
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    dims = (16, 16, 16)
    L, _, _, _ = oracle.hierarchy(*dims, varcoef=(2, 0.5))
    n = L[0].nrow
    ref = RefProblem(*dims)
    for l, lev in enumerate(L):
        ref.set_level_values(l, lev.vals)
    b = oracle.uniform(3, n)
    r = oracle.uniform(12, n)
    assert (oracle.mg(L, r) == ref.mg(r)).all()
    x1, k1, nr1, nr01 = oracle.cg(L, b, np.zeros(n), 500, 1e-12)
    x2, k2, nr2, nr02, _ = ref.cg(b, np.zeros(n), 500, 1e-12)
    assert k1 == k2 and np.abs(x1 - x2).max() < 1e-12
    ref.close()


@pytest.mark.parametrize("dims", [(16, 16, 16), (16, 24, 32), (24, 24, 24), (10, 6, 14)],
                         ids=lambda d: "x".join(map(str, d)))
def test_matrix_free_restatements_match_stored(dims, oracle):
    """The matrix-free SpMV / colour-ordered SYMGS (FP64 and the mixed FP32/BF16
    sweep) that check benchmark-size grids are bit-identical to the stored-matrix
    restatements pinned above, on even, odd and non-cubic grids."""
    L, b, x, xe = oracle.hierarchy(*dims, levels=1)
    oracle.colour_order(L)
    lev = L[0]
    u, r, x0 = inputs(oracle, lev.nrow)
    assert (oracle.stencil_spmv(dims, u) == oracle.spmv(lev, u)).all()
    assert (oracle.stencil_symgs(dims, r, x0) == oracle.symgs(lev, r, x0, coloured=True)).all()
    x32 = x0.astype(np.float32)
    assert (oracle.stencil_symgs32(dims, r, x32) == oracle.symgs32(lev, r, x32)).all()
    # and against the reference's own ComputeSPMV_ref on the same grid
    from oracle.oracle import RefProblem
    if RefProblem.available() and all(d % 8 == 0 for d in dims):   # its 4-level hierarchy
        R = RefProblem(*dims)
        try:
            assert (oracle.stencil_spmv(dims, u) == R.spmv(0, u)).all()
        finally:
            R.close()


def test_bf16_rounding_against_torch(oracle):
    """The FP64 -> BF16 conversion of the mixed V-cycle's values (through
    FP32, nearest-even at each step) equals torch's float64 -> float32 ->
    bfloat16 conversion: random magnitudes, exact ties in both parities,
    FP32 subnormals, signed zeros and infinities; a NaN stays a NaN (its bit
    pattern is each implementation's own)."""
    rng = np.random.default_rng(7)
    v = np.concatenate([
        rng.standard_normal(20000) * 10.0 ** rng.integers(-40, 39, 20000),
        -np.exp(0.5 * rng.standard_normal(5000)),               # variable-coefficient values
        [0.0, -0.0, np.inf, -np.inf, np.nan, 26.0, -1.0, 1e-45, -1e-44, 3.4e38, 1e39],
    ])
    # FP32 values halfway between two BF16 values, with even and odd BF16 lsb
    hi = rng.integers(0, 0x7f7f, 4000, dtype=np.uint32) << 16
    ties = (hi | 0x8000).view(np.float32).astype(np.float64)
    v = np.concatenate([v, ties, -ties])
    import torch
    lib = oracle.lib()
    got = np.array([lib.or_bf16_from_double(float(x)) for x in v], dtype=np.uint16)
    want = torch.from_numpy(v).to(torch.float32).to(torch.bfloat16).view(torch.int16).numpy()
    nan = np.isnan(v)
    assert (got[~nan] == want.view(np.uint16)[~nan]).all()
    assert ((got[nan] & 0x7f80) == 0x7f80).all() and ((got[nan] & 0x7f) != 0).all()
