"""The sharded (z-slab) solver on the GPU, through the C ABI.

* In-process groups of 2 and 4 slabs on one GPU (hpcgx_group_*) against the
  oracle's restatement of the multi-rank algorithm (Oracle.slab_hierarchy,
  itself checked against per-rank halo exchange over gloo in
  test_sharded_cpu.py): SpMV, SYMGS and the V-cycle bit-exact on every level;
  CG to 1e-10 with the oracle's iteration count (dot products round
  differently, as in the one-GPU tests); the mixed solver to the FP64 target.
* The NCCL backend with one rank, and a group of one slab: both run the
  sharded step sequence (separate restriction / prolongation launches,
  deferred reductions summed over the ranks) and must reproduce the fused
  one-GPU solver bit for bit.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [((16, 8, 8), 2), ((8, 16, 8), 4), ((16, 16, 16), 2)]


def ids(c):
    return "%dx%dx%d_x%d" % (c[0] + (c[1],))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


_cache = {}


def setup(case, oracle):
    if case in _cache:
        return _cache[case]
    from hpcg_b200 import Group, Problem
    (nx, ny, nz), P = case
    L, _, _, _ = oracle.slab_hierarchy(nx, ny, nz, P)
    oracle.colour_order(L)
    ranks = [Problem(nx, ny, nz, nranks=P, rank=r) for r in range(P)]
    for p in ranks:
        p.generate("hpcg")
    g = Group(ranks)
    _cache[case] = (L, ranks, g)
    return _cache[case]


def split(v, P):
    return [cuda(c) for c in np.split(v, P)]


def join(ts):
    return np.concatenate([host(t) for t in ts])


@pytest.fixture(scope="module", params=CASES, ids=ids)
def case(request):
    return request.param


def test_group_operators_bitexact(case, oracle):
    L, ranks, g = setup(case, oracle)
    P = len(ranks)
    for l, lev in enumerate(L):
        n = lev.nrow
        u, r, x0 = (oracle.uniform(s, n) for s in (11, 12, 13))
        assert (join(g.spmv(split(u, P), level=l)) == oracle.spmv(lev, u)).all()
        xs = split(x0, P)
        g.symgs(split(r, P), xs, level=l)
        assert (join(xs) == oracle.symgs(lev, r, x0, coloured=True)).all()
    r = oracle.uniform(12, L[0].nrow)
    assert (join(g.mg(split(r, P))) == oracle.mg(L, r, coloured=True)).all()


def test_group_cg(case, oracle):
    from hpcg_b200._lib import CG_MG, CG_MIXED, CG_PLAIN
    L, ranks, g = setup(case, oracle)
    P = len(ranks)
    n = L[0].nrow
    u = oracle.uniform(1, n, -1.0, 1.0)
    b = oracle.spmv(L[0], u)
    for mode, precond in ((CG_MG, True), (CG_PLAIN, False)):
        xs = split(np.zeros(n), P)
        k, nr, nr0 = g.cg(split(b, P), xs, 500, 1e-10, mode=mode)
        ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 500, 1e-10, precond=precond,
                                      coloured=True)
        assert k == ok and nr / nr0 <= 1e-10
        assert np.abs(join(xs) - ox).max() <= 1e-8 * np.abs(ox).max()
    # ten iterations: residual trajectory within 1e-8 relative
    xs = split(np.zeros(n), P)
    k, nr, nr0 = g.cg(split(b, P), xs, 10, 0.0, mode=CG_MG)
    ox, ok, onr, onr0 = oracle.cg(L, b, np.zeros(n), 10, 0.0, precond=True, coloured=True)
    assert k == ok == 10 and abs(nr / onr - 1.0) < 1e-8
    # mixed precision over the slabs: the oracle's flexible CG on the same
    # decomposition, the FP64 target, the true residual honest
    for p in ranks:
        p.build_mixed()
    xs = split(np.zeros(n), P)
    k, nr, nr0 = g.cg(split(b, P), xs, 500, 1e-10, mode=CG_MIXED)
    ox, ok, onr, onr0 = oracle.fcg(L, b, np.zeros(n), 500, 1e-10)
    assert k == ok and nr / nr0 <= 1e-10
    x = join(xs)
    assert np.linalg.norm(b - oracle.spmv(L[0], x)) / np.linalg.norm(b) < 1e-9


def test_one_rank_sharded_paths_reproduce_fused_solver(oracle):
    """A group of one slab and the NCCL backend with one rank run the step
    sequence of the sharded solver; both must equal the fused solver."""
    from hpcg_b200 import Group, Problem, nccl_unique_id
    dims = (16, 16, 16)
    ref = Problem(*dims)
    ref.generate("hpcg")
    ref.build_mixed()
    n = ref.rows()
    u = ref.fill_uniform(1, -1.0, 1.0)
    b = ref.spmv(u)
    want = {}
    for name, f in (("mg", lambda P, x: P.cg(b, x, 500, 1e-10)),
                    ("mixed", lambda P, x: P.cg_mixed(b, x, 500, 1e-10))):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        want[name] = (f(ref, x), host(x))
    r = ref.fill_uniform(12, 0.0, 1.0)
    want_mg = host(ref.mg(r))

    one = Problem(*dims, nranks=1, rank=0)
    one.generate("hpcg")
    one.build_mixed()
    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")   # one rank: no peer to reach
    one.attach_nccl(nccl_unique_id())
    for name, f in (("mg", lambda P, x: P.cg(b, x, 500, 1e-10)),
                    ("mixed", lambda P, x: P.cg_mixed(b, x, 500, 1e-10))):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        got = f(one, x)
        assert got == want[name][0]
        assert (host(x) == want[name][1]).all()
    assert (host(one.mg(r)) == want_mg).all()
    assert (host(one.spmv(u)) == host(b)).all()
    one.close()

    solo = Problem(*dims, nranks=1, rank=0)
    solo.generate("hpcg")
    g = Group([solo])
    xs = [torch.zeros(n, dtype=torch.float64, device="cuda")]
    from hpcg_b200._lib import CG_MG
    got = g.cg([b], xs, 500, 1e-10, mode=CG_MG)
    assert got == want["mg"][0]
    assert (host(xs[0]) == want["mg"][1]).all()
    assert (host(g.mg([r])[0]) == want_mg).all()
    g.close()
    solo.close()
    ref.close()


def test_group_checks_its_ranks(oracle):
    from hpcg_b200 import Group, HPCGXError, Problem
    a = Problem(16, 16, 8, nranks=2, rank=0)
    b = Problem(16, 16, 8, nranks=2, rank=1)
    c = Problem(16, 8, 8, nranks=2, rank=1)
    with pytest.raises(HPCGXError):
        Group([b, a])                  # rank r must sit at position r
    with pytest.raises(HPCGXError):
        Group([a, c])                  # slabs of different geometry
    with pytest.raises(HPCGXError):
        Group([a])                     # slab 0 of 2 alone
    for p in (a, b, c):
        p.close()


def test_sharded_problem_needs_a_backend(oracle):
    from hpcg_b200 import HPCGXError, Problem
    p = Problem(16, 16, 8, nranks=2, rank=1)
    p.generate("hpcg")
    n = p.rows()
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(HPCGXError):
        p.cg(b, x, 10, 0.0)
    with pytest.raises(HPCGXError):
        p.generate("varcoef", seed=2, sigma=1.0)
    p.close()


_STALL_SCRIPT = r"""
import os, sys, torch
sys.path.insert(0, os.environ["HPCGX_ROOT"])
from hpcg_b200 import HPCGXError, Problem, nccl_unique_id
dims = (16, 16, 16)
ref = Problem(*dims)
ref.generate("hpcg")
u = ref.fill_uniform(1, -1.0, 1.0)
b = ref.spmv(u)
x = torch.zeros_like(b)
want = ref.cg(b, x, 500, 1e-10)
one = Problem(*dims, nranks=1, rank=0)
one.generate("hpcg")
try:
    one.attach_nccl(nccl_unique_id())
    raise SystemExit("the stalled communicator was not reported")
except HPCGXError as e:
    assert e.code == 8, e                      # HPCGX_ETIMEOUT
    assert "aborted" in str(e), e
# the problem stays usable; a new communicator replaces the aborted one
one.attach_nccl(nccl_unique_id())
x.zero_()
got = one.cg(b, x, 500, 1e-10)
assert got == want, (got, want)
one.close()
ref.close()
print("stall-ok")
"""


def test_nccl_stall_times_out_and_aborts(tmp_path):
    """A communicator that never settles (a peer that has died, faked on the
    host with HPCGX_FAULT_NCCL_STALL: the first settle of the process sees
    ncclInProgress for ever) is aborted after HPCGX_WAIT_TIMEOUT_S and the call
    returns HPCGX_ETIMEOUT; the problem stays usable and a new communicator
    solves as before.  One rank, so no kernel ever waits for another."""
    import subprocess
    import sys
    from conftest import ROOT
    # the limit must leave a real communicator time to initialise (about a
    # second); the faked stall then waits it out once
    env = dict(os.environ, HPCGX_ROOT=ROOT, HPCGX_WAIT_TIMEOUT_S="10",
               HPCGX_FAULT_NCCL_STALL="1", NCCL_SOCKET_IFNAME="lo", NCCL_NVLS_ENABLE="0")
    script = tmp_path / "stall.py"
    script.write_text(_STALL_SCRIPT)
    out = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0 and "stall-ok" in out.stdout, out.stdout + out.stderr[-3000:]
