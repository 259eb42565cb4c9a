"""Generates the golden vectors in tests/golden/ by running the reference itself.

Every array in the fixtures is an output of the reference's own code
(src/*_ref.cpp, CG_ref, GenerateProblem_ref, ...) compiled from its sources by
oracle/Makefile into oracle/_ref/libhpcgref.so, on seeded inputs:

  u  = uniform[1, 2)  (SplitMix64 draws, seed 11)   x-like input
  r  = uniform[0, 1)  (seed 12)                      right-hand side
  x0 = uniform[0, 1)  (seed 13)                      Gauss-Seidel start

The colour-permuted entries use ComputeSYMGS_ref / ComputeMG_ref / CG_ref on
the matrix permuted by the greedy colouring order (src/OptimizeProblem.cpp
:43-96, restated in the oracle).  Rerun with the reference sources present:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle, RefProblem, build  # noqa: E402

GRIDS = [(16, 16, 16), (16, 24, 32)]


def fixture_name(dims):
    return os.path.join(HERE, "ref_%dx%dx%d.npz" % dims)


def make(dims):
    ref = RefProblem(*dims)
    L, _, _, _ = Oracle.hierarchy(*dims)
    Oracle.colour_order(L)
    ref.build_permuted([lev.position for lev in L])
    n = ref.rows(0)
    out = {"dims": np.array(dims)}
    b, x, xexact = ref.vectors()
    out["b"] = b
    u = Oracle.uniform(11, n, 1.0, 2.0)
    r = Oracle.uniform(12, n)
    x0 = Oracle.uniform(13, n)
    for l in range(4):
        nl = ref.rows(l)
        out["spmv_L%d" % l] = ref.spmv(l, u[:nl].copy())
        out["symgs_perm_L%d" % l] = ref.symgs_permuted(l, r[:nl].copy(), x0[:nl].copy())
    out["symgs_L0"] = ref.symgs(0, r, x0)
    out["mg"] = ref.mg(r)
    out["mg_perm"] = ref.mg_permuted(r)
    # restriction / prolongation of level 0 -> 1 on seeded inputs
    nc = ref.rows(1)
    out["restriction_L0"] = ref.restriction(0, r, u)
    out["prolongation_L0"] = ref.prolongation(0, u[:nc].copy(), x0)
    out["dot_ur"] = np.array([ref.dot(u, r)])
    out["dot_uu"] = np.array([ref.dot(u, u)])
    out["waxpby_a1"] = ref.waxpby(1.0, u, 0.37, r)
    out["waxpby_b1"] = ref.waxpby(-0.61, u, 1.0, r)
    out["waxpby_ab"] = ref.waxpby(0.83, u, -1.29, r)
    out["residual_ur"] = np.array([ref.residual(u, r)])
    # A * xexact = b exactly (src/TestSymmetry.cpp:122-132)
    out["A_xexact_resid"] = np.array([ref.residual(ref.spmv(0, xexact), b)])
    # CG_ref: 10 iterations (trajectory) and to 1e-10 (iteration count)
    for tag, it, tol in (("cg10", 10, 0.0), ("cgtol", 500, 1e-10)):
        xs, k, nr, nr0, _ = ref.cg(b, np.zeros(n), it, tol)
        out[tag + "_x"], out[tag + "_stats"] = xs, np.array([k, nr, nr0])
        xs, k, nr, nr0 = ref.cg_permuted(b, np.zeros(n), it, tol)
        out[tag + "_perm_x"], out[tag + "_perm_stats"] = xs, np.array([k, nr, nr0])
    # TestCG (src/TestCG.cpp:62-111): diagonal x1e6 (rows with id < 9 get
    # (id+2)*1e6), b scaled alike; iteration counts of unpreconditioned and
    # preconditioned CG to 1e-12.
    d = np.full(n, 26.0)
    scale = np.full(n, 1.0e6)
    scale[:9] = (np.arange(9) + 2) * 1.0e6
    ref.replace_diagonal(0, d * scale)
    bs = b * scale
    for tag, prec in (("testcg_noprec", False), ("testcg_prec", True)):
        _, k, nr, nr0, _ = ref.cg(bs, np.zeros(n), 50, 1e-12, precond=prec)
        out[tag] = np.array([k, nr, nr0])
    ref.replace_diagonal(0, d)
    ref.close()
    np.savez_compressed(fixture_name(dims), **out)
    return out


def main():
    build()
    if not RefProblem.available():
        raise SystemExit("oracle/_ref/libhpcgref.so missing: the reference sources are needed")
    for dims in GRIDS:
        out = make(dims)
        print(fixture_name(dims), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
