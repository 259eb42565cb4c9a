"""The differentiable solve x = A(vals)^{-1} b (hpcg_b200.solve).

* 128^3 variable-coefficient problem (a_ij = -exp(0.5 z), z ~ N(0,1) per edge,
  seed 2; b ~ U(0,1) and x_target ~ N(0,1), seed 3; L = 1/2 |x - x_target|^2):
  FP64 forward and adjoint MG-PCG to 1e-12; the gradient with respect to b and
  all 27 values per row is checked against central finite differences on 16
  random edge-symmetric directions (seed 4), relative error <= 1e-6.
* Against a CPU reference gradient built from the reference's own CG_ref
  (oracle/_ref) on the same matrix: relative error <= 1e-8.
* Mixed precision (FP32/BF16 V-cycle in FP64 flexible CG) forward + adjoint
  to 1e-10: gradient within 1e-6 of the FP64 adjoint gradient.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def loss_parts(x, xt):
    return 0.5 * torch.sum((x - xt) ** 2)


def test_fd_gradient_128():
    from hpcg_b200 import solve, symmetric_direction, varcoef_problem
    P, vals = varcoef_problem(128, 128, 128, seed=2, sigma=0.5)
    n = P.rows()
    b = P.fill_uniform(3, 0.0, 1.0)
    xt = P.fill_normal(3, offset=n)
    v = vals.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    x = solve(v, bb, P, tol=1e-12)
    L = loss_parts(x, xt)
    L.backward()
    gv, gb = v.grad, bb.grad
    xs = x.detach()
    g = torch.Generator(device="cuda").manual_seed(4)
    worst = 0.0
    for _ in range(16):
        Dv = symmetric_direction(P, g) * vals.abs()
        Db = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
        h = 1e-5
        dl = []
        for sgn in (1.0, -1.0):
            P.set_values((vals + sgn * h * Dv).reshape(-1), level=0, recoarsen=True)
            xp = xs.clone()                       # warm start from the base solution
            k, nr, nr0 = P.cg(b + sgn * h * Db, xp, 2000, 1e-11)
            d = xp - xs
            dl.append(torch.sum(d * (xs - xt + 0.5 * d)).item())
        fd = (dl[0] - dl[1]) / (2 * h)
        an = (torch.sum(gv * Dv) + torch.sum(gb * Db)).item()
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst <= 1e-6, worst


def test_gradient_matches_cg_ref(oracle):
    from oracle.oracle import RefProblem
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built")
    from hpcg_b200 import Problem, solve
    dims = (32, 32, 32)
    L, _, _, _ = oracle.hierarchy(*dims, varcoef=(2, 0.5))
    n = L[0].nrow
    b = oracle.uniform(3, n)
    xt = oracle.normal(3, 2 * n)[n:]
    ref = RefProblem(*dims)
    for l, lev in enumerate(L):
        ref.set_level_values(l, lev.vals)
    x_ref, k1, _, _, _ = ref.cg(b, np.zeros(n), 500, 1e-13)
    lam_ref, k2, _, _, _ = ref.cg(x_ref - xt, np.zeros(n), 500, 1e-13)
    g_ref = oracle.adjoint_grad(L[0], lam_ref, x_ref).reshape(n, 27)
    ref.close()
    # the same matrix on the GPU, loaded from the host values
    P = Problem(*dims)
    for l, lev in enumerate(L):
        P.load_level(l, lev.nnz, lev.cols, lev.vals)
    vals, cols = P.get_values(0)
    v = vals.clone().requires_grad_(True)
    bb = torch.from_numpy(b).cuda().requires_grad_(True)
    x = solve(v, bb, P, tol=1e-13)
    loss_parts(x, torch.from_numpy(xt).cuda()).backward()
    # packed (reference entry order) -> stencil slots
    g = v.grad.cpu().numpy()
    c = cols.cpu().numpy()
    gp = np.zeros_like(g_ref)
    rows = np.arange(n)
    for j in range(27):
        m = j < L[0].nnz
        col = L[0].cols[rows * 27 + j]
        dx = col % 32 - rows % 32
        dy = (col // 32) % 32 - (rows // 32) % 32
        dz = col // 1024 - rows // 1024
        s = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)
        gp[m, j] = g[rows[m], s[m]]
        assert (c[rows[m], s[m]] == col[m]).all()
    err = np.linalg.norm(gp - g_ref) / np.linalg.norm(g_ref)
    assert err <= 1e-8, err
    assert np.linalg.norm(bb.grad.cpu().numpy() - lam_ref) / np.linalg.norm(lam_ref) <= 1e-8


def test_mixed_adjoint_matches_fp64():
    from hpcg_b200 import solve, varcoef_problem
    P, vals = varcoef_problem(128, 128, 64, seed=5, sigma=1.0)
    n = P.rows()
    b = P.fill_uniform(6, 0.0, 1.0)
    xt = P.fill_normal(6, offset=n)
    grads = []
    for mixed in (False, True):
        v = vals.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        x = solve(v, bb, P, tol=1e-10, mixed=mixed)
        loss_parts(x, xt).backward()
        grads.append((v.grad, bb.grad))
    e_v = (torch.linalg.norm(grads[1][0] - grads[0][0]) / torch.linalg.norm(grads[0][0])).item()
    e_b = (torch.linalg.norm(grads[1][1] - grads[0][1]) / torch.linalg.norm(grads[0][1])).item()
    assert e_v <= 1e-6 and e_b <= 1e-6, (e_v, e_b)


def test_solve_input_checks():
    from hpcg_b200 import solve, varcoef_problem
    P, vals = varcoef_problem(16, 16, 16, seed=1, sigma=0.5)
    b = torch.ones(P.rows(), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        solve(vals[:-1], b, P)
    with pytest.raises(TypeError):
        solve(vals.float(), b.float(), P)
