"""The index-checked build on the GPU: every kernel family runs on small and
odd grids, one rank and sharded, and no kernel may meet an out-of-range
storage row, vector row or column (libhpcgx_checked.so records the first one
and redirects the access into the buffers; hpcgx_check_status reports it).
This stands in for a memory checker, which this GPU pool does not run.
The checked library is loaded in a child process (HPCGX_LIBRARY=checked is
read when the library is first loaded)."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 16), (24, 24, 24), (16, 24, 32), (64, 32, 16)]


def _run(rank, out):
    import sys
    os.environ["HPCGX_LIBRARY"] = "checked"
    sys.path.insert(0, ROOT)
    torch.cuda.set_device(0)
    import hpcg_b200._lib as L
    assert L.LIB_PATH.endswith("libhpcgx_checked.so")
    from hpcg_b200 import Group, Problem, check_status
    done = []
    for dims in GRIDS:
        P = Problem(*dims)
        P.generate("hpcg")
        P.build_mixed()
        n = P.rows()
        u = P.fill_uniform(1, -1.0, 1.0)
        b = P.spmv(u)
        for l in range(4):
            ul = u[:P.rows(l)].clone()
            P.spmv(ul, level=l)
            P.spmv(ul, level=l, stencil_cols=True)
            x = torch.zeros_like(ul)
            P.symgs(ul, x, level=l)
            P.spmv_mixed(ul.float(), level=l)
            x32 = torch.zeros(P.rows(l), dtype=torch.float32, device="cuda")
            P.symgs_mixed(ul if l == 0 else ul.float(), x32, level=l)
        P.mg(b)
        P.mg_mixed(b)
        for f in (lambda x: P.cg(b, x, 60, 1e-10), lambda x: P.cg(b, x, 30, 0.0, precond=False),
                  lambda x: P.cg_mixed(b, x, 60, 1e-10)):
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            f(x)
        check_status()
        done.append(("one rank", dims))
        P.close()
    # variable coefficients and the adjoint gradient
    from hpcg_b200 import varcoef_problem
    P, vals = varcoef_problem(16, 16, 16, seed=2, sigma=0.5)
    n = P.rows()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    P.cg(torch.ones(n, dtype=torch.float64, device="cuda"), x, 60, 1e-10)
    P.adjoint_grad(torch.ones_like(x), x)
    check_status()
    done.append(("varcoef", (16, 16, 16)))
    # sharded groups
    for (dims, ranks) in (((16, 8, 8), 2), ((8, 16, 8), 4)):
        ps = [Problem(*dims, nranks=ranks, rank=r) for r in range(ranks)]
        for p in ps:
            p.generate("hpcg")
            p.build_mixed()
        g = Group(ps)
        m = ps[0].rows()
        xs = [torch.rand(m, dtype=torch.float64, device="cuda") for _ in ps]
        for l in range(4):
            g.spmv([x[:ps[0].rows(l)].contiguous() for x in xs], level=l)
            g.symgs([x[:ps[0].rows(l)].contiguous() for x in xs],
                    [torch.zeros(ps[0].rows(l), dtype=torch.float64, device="cuda") for _ in ps],
                    level=l)
        g.mg(xs)
        for mode in (0, 1, 2):
            g.cg(xs, [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in ps], 40, 1e-10,
                 mode=mode)
        check_status()
        done.append(("group", dims, ranks))
        g.close()
    out["done"] = done


def test_checked_build_meets_no_bad_index():
    if not os.path.exists(os.path.join(ROOT, "hpcg_b200", "libhpcgx_checked.so")):
        pytest.skip("libhpcgx_checked.so not built")
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_run, args=(out,), nprocs=1, join=True, start_method="spawn")
    assert len(out["done"]) == len(GRIDS) + 3
