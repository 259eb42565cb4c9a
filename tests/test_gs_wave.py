"""The one-launch symmetric sweep (k_gs_wave) against the seven class launches.

k_gs_wave runs the seven class steps of a symmetric Gauss-Seidel sweep as a
wavefront over the z-planes inside one launch; within a colour the rows are
independent, so every result must be bit-identical to the class launches
(``==``): SYMGS on every level, both V-cycles, both solvers (same iteration
counts and the same x), sharded groups included.  The schedule is stressed
with the smallest stage lag (2 planes) and one-line work items, which
maximise the number of waits, as well as the default and a long lag.
HPCGX_GS_WAVE / HPCGX_WAVE_LAG / HPCGX_WAVE_ROWS are read when a problem is
created (the class launches are the default).
"""
import os

import pytest
import torch

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 16), (24, 24, 24), (16, 24, 32), (64, 32, 16), (32, 32, 64)]
SCHEDULES = {"lag2-line": {"HPCGX_WAVE_LAG": "2", "HPCGX_WAVE_ROWS": "1"},
             "default": {},
             "lag9-64rows": {"HPCGX_WAVE_LAG": "9", "HPCGX_WAVE_ROWS": "64"}}


def _make(dims, env, **kw):
    from hpcg_b200 import Problem
    keys = ["HPCGX_GS_WAVE", "HPCGX_WAVE_LAG", "HPCGX_WAVE_ROWS"]
    old = {k: os.environ.get(k) for k in keys}
    try:
        for k in keys:
            os.environ.pop(k, None)
        os.environ.update(env)
        P = Problem(*dims, **kw)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    P.generate("hpcg")
    P.build_mixed()
    return P


def _same(a, b):
    return torch.equal(a, b)


@pytest.mark.parametrize("sched", list(SCHEDULES), ids=list(SCHEDULES))
@pytest.mark.parametrize("dims", GRIDS, ids=lambda d: "x".join(map(str, d)))
def test_one_launch_sweep_matches_class_launches(dims, sched):
    from hpcg_b200 import check_status
    Pc = _make(dims, {"HPCGX_GS_WAVE": "0"})
    Pw = _make(dims, {"HPCGX_GS_WAVE": "1", **SCHEDULES[sched]})
    n = Pc.rows()
    u = Pc.fill_uniform(1, -1.0, 1.0)
    b = Pc.spmv(u)
    for l in range(4):
        m = Pc.rows(l)
        r = u[:m].clone()
        x0 = torch.rand(m, dtype=torch.float64, device="cuda")
        xc, xw = x0.clone(), x0.clone()
        Pc.symgs(r, xc, level=l)
        Pw.symgs(r, xw, level=l)
        assert _same(xc, xw), "SYMGS level %d" % l
        r32 = r if l == 0 else r.float()
        x32 = x0.float()
        xc32, xw32 = x32.clone(), x32.clone()
        Pc.symgs_mixed(r32, xc32, level=l)
        Pw.symgs_mixed(r32, xw32, level=l)
        assert _same(xc32, xw32), "mixed SYMGS level %d" % l
    assert _same(Pc.mg(b), Pw.mg(b))
    assert _same(Pc.mg_mixed(b), Pw.mg_mixed(b))
    for solve in ("cg", "cg_mixed"):
        xc = torch.zeros(n, dtype=torch.float64, device="cuda")
        xw = torch.zeros(n, dtype=torch.float64, device="cuda")
        kc = getattr(Pc, solve)(b, xc, 60, 1e-10)
        kw = getattr(Pw, solve)(b, xw, 60, 1e-10)
        assert kc[0] == kw[0] and kc[1] == kw[1], solve
        assert _same(xc, xw), solve
    check_status()
    Pc.close()
    Pw.close()


@pytest.mark.parametrize("dims,ranks", [((16, 8, 8), 2), ((8, 16, 8), 4), ((32, 16, 16), 2)])
def test_one_launch_sweep_in_sharded_groups(dims, ranks):
    from hpcg_b200 import Group, check_status
    runs = {}
    for wave in ("0", "1"):
        env = {"HPCGX_GS_WAVE": wave, "HPCGX_WAVE_LAG": "2", "HPCGX_WAVE_ROWS": "1"}
        ps = [_make(dims, env, nranks=ranks, rank=r) for r in range(ranks)]
        g = Group(ps)
        m = ps[0].rows()
        gen = torch.Generator(device="cuda").manual_seed(5)
        rs = [torch.rand(m, dtype=torch.float64, device="cuda", generator=gen) for _ in ps]
        sweeps = []
        for l in range(4):   # level 3 of the first two cases has ny or nz = 1: class launches
            ml = ps[0].rows(l)
            xl = [v[:ml].clone() for v in rs]
            g.symgs([v[:ml].contiguous() for v in rs], xl, level=l)
            sweeps += xl
        mg = [v.clone() for v in g.mg(rs)] + sweeps
        xs = [torch.zeros(m, dtype=torch.float64, device="cuda") for _ in ps]
        k = g.cg(rs, xs, 40, 1e-10)
        runs[wave] = (mg, k, xs)
        check_status()
        g.close()
    (mg0, k0, x0), (mg1, k1, x1) = runs["0"], runs["1"]
    assert all(_same(a, b) for a, b in zip(mg0, mg1))
    assert k0 == k1
    assert all(_same(a, b) for a, b in zip(x0, x1))
