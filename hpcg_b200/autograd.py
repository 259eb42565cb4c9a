"""Differentiable solve x = A(vals)^{-1} b on the GPU (no reference counterpart).

``solve(vals, b, problem)`` is a torch.autograd.Function over the same C ABI
as the benchmark path.  ``vals`` holds the finest-level matrix in natural row
order with the 27 stencil slots of each row (slot (dz+1)*9+(dy+1)*3+(dx+1);
slots without a neighbour are ignored), and must describe a symmetric
positive definite matrix (a_ij = a_ji).

Forward: the values are written to the device (coarse levels are rebuilt from
them for the preconditioner), and MG-PCG solves A x = b (FP64, or the FP32/BF16
V-cycle inside FP64 flexible CG with ``mixed=True``).  x is kept for the
backward pass, not recomputed.

Backward: A is symmetric, so the adjoint system A lambda = dL/dx is solved on
the same MG-PCG kernels; dL/db = lambda and dL/dvals_ij = -lambda_i x_j, the
latter by the stencil-pattern sampled-outer-product kernel (hpcgx_adjoint_grad).
"""
from __future__ import annotations

import torch

from .problem import STENCIL, Problem


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, b, problem, tol, max_iter, mixed):
        problem.set_values(vals.reshape(-1), level=0, recoarsen=True)
        b = b.contiguous()
        x = torch.zeros_like(b)
        f = problem.cg_mixed if mixed else problem.cg
        k, nr, nr0 = f(b, x, max_iter, tol)
        if not nr <= tol * nr0:
            raise RuntimeError(f"forward solve stopped at {nr / nr0:.3e} after {k} iterations")
        ctx.problem, ctx.tol, ctx.max_iter, ctx.mixed = problem, tol, max_iter, mixed
        ctx.version = problem.values_version
        ctx.save_for_backward(vals, x)
        ctx.stats = (k, nr / nr0)
        return x

    @staticmethod
    def backward(ctx, gx):
        vals, x = ctx.saved_tensors
        P = ctx.problem
        if P.values_version != ctx.version:      # the problem was reused since forward
            P.set_values(vals.reshape(-1), level=0, recoarsen=True)
            ctx.version = P.values_version
        gx = gx.contiguous()
        lam = torch.zeros_like(x)
        if torch.count_nonzero(gx) > 0:
            f = P.cg_mixed if ctx.mixed else P.cg
            k, nr, nr0 = f(gx, lam, ctx.max_iter, ctx.tol)
            if not nr <= ctx.tol * nr0:
                raise RuntimeError(f"adjoint solve stopped at {nr / nr0:.3e} after {k} iterations")
        gvals = P.adjoint_grad(lam, x) if ctx.needs_input_grad[0] else None
        gb = lam if ctx.needs_input_grad[1] else None
        return gvals, gb, None, None, None, None


def solve(vals: torch.Tensor, b: torch.Tensor, problem: Problem, tol: float = 1e-12,
          max_iter: int = 2000, mixed: bool = False) -> torch.Tensor:
    """x = A(vals)^{-1} b; differentiable in vals ((n, 27) float64) and b ((n,) float64)."""
    n = problem.rows(0)
    if vals.shape != (n, STENCIL) or b.shape != (n,):
        raise ValueError(f"vals must be ({n}, {STENCIL}) and b ({n},)")
    if vals.dtype != torch.float64 or b.dtype != torch.float64:
        raise TypeError("vals and b must be float64")
    return _Solve.apply(vals, b, problem, tol, max_iter, mixed)


def varcoef_problem(nx, ny, nz, seed, sigma, levels=4, device=0):
    """A problem holding the variable-coefficient matrix a_ij = -exp(sigma z_ij),
    z ~ N(0,1) per edge, diagonal sum|a_ij| + 2, and its values as a (n, 27)
    tensor suitable for ``solve``."""
    P = Problem(nx, ny, nz, levels=levels, device=device)
    P.generate("varcoef", seed=seed, sigma=sigma)
    vals, _ = P.get_values(0)
    return P, vals.clone()


def symmetric_direction(problem: Problem, generator: torch.Generator) -> torch.Tensor:
    """A random (n, 27) direction with D_ij = D_ji (edge-symmetric, so A + h D
    stays symmetric), zero where the stencil has no neighbour."""
    nx, ny, nz = problem.level_dims(0)
    n = nx * ny * nz
    dev = problem.device
    D = torch.randn(n, STENCIL, dtype=torch.float64, device=dev, generator=generator)
    row = torch.arange(n, device=dev)
    ix, iy, iz = row % nx, (row // nx) % ny, row // (nx * ny)
    out = torch.zeros_like(D)
    for s in range(STENCIL):
        dx, dy, dz = s % 3 - 1, (s // 3) % 3 - 1, s // 9 - 1
        ok = ((ix + dx >= 0) & (ix + dx < nx) & (iy + dy >= 0) & (iy + dy < ny) &
              (iz + dz >= 0) & (iz + dz < nz))
        if s >= 13:
            out[:, s] = torch.where(ok, D[:, s], 0.0)
        else:
            # the reverse edge of (row, s) is (row + off(s), 26 - s): copy its draw
            nb = row + dz * nx * ny + dy * nx + dx
            src = torch.where(ok, nb, row)
            out[:, s] = torch.where(ok, D[src, 26 - s], 0.0)
    return out
