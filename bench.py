"""Benchmark: time to FP64 relative residual 1e-10, mixed vs FP64 PCG, on B200.

Workload (one "step" = one solve): the HPCG 27-point problem on a 512^3 grid
(134M rows, 3.6e9 nonzeros), 4-level multigrid, 8-colour Gauss-Seidel;
b = A u with u ~ U(-1, 1) (SplitMix64 seed 1), x0 = 0; solved to
||r||/||r0|| <= 1e-10 by the mixed-precision flexible PCG (FP32/BF16 V-cycle
inside FP64 CG).  The plain FP64 PCG solve of the same system is timed beside
it for the mixed-vs-FP64 comparison.  Inputs are generated on the device
(synthetic, as HPCG generates its own problem).

  value        seconds per mixed solve (mean of --steps timed solves), lower is better
  e2e          the same through the C ABI from pinned host buffers (b and x0
               copied in, x copied out inside the timed region)
  roofline     the largest kernel, the mixed solver's FP64 SpMV (and, beside
               it, the finest-level Gauss-Seidel class kernels): algorithmic
               bytes / CUDA-event duration of every launch in the timed region,
               against the measured HBM copy bandwidth
  cpu_baseline the reference's own CG_ref (oracle/_ref, OpenMP on all host
               cores): the per-iteration time of a few iterations on a 256^3
               sample of the same problem (b = A u), scaled x8 in rows to
               512^3 and to the reference's own (natural-order) iteration
               count to 1e-10, measured at 32^3 - 256^3 and extrapolated to
               512^3 (the reference's int32 counters overflow there)

Multi-GPU (torchrun, N ranks): one system of N z-slabs, each GPU holding one
512^3 slab (weak scaling; the reference's 1 x 1 x N process grid): halo planes
are exchanged and dot products summed over NCCL, the smoother is block Jacobi
across slabs as in the reference, so the iteration count depends on N.  value
is the max over ranks of the solve time.  --replicas runs N independent
systems instead.  The sharded solver runs step by step without CUDA graphs,
so the per-kernel probes (roofline) are reported at N = 1 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to FP64 rel. residual 1e-10, mixed vs FP64 PCG on 1 B200; GFLOP/s; HBM %"
TOL = 1e-10
MAX_IT = 2000
SEED_U = 1
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def model(dims, levels=4):
    """HPCG's flop model (src/ReportResults.cpp:81-97) and the reference
    implementation's bytes per iteration: SpMV 12 nnz + 16 n, SYMGS 24 nnz + 48 n,
    R+P 40 n_c, CG vectors 112 n (FP64; three dot products and three WAXPBYs of
    src/CG.cpp:100-130); for the mixed solver the same steps with 6 B/nnz in the
    V-cycle (BF16 value + int32 column) and FP32 vectors.  This design moves less
    than either (restriction and prolongation inside the sweeps, zero-guess
    sweeps, values-only BF16 matrix, columns from the stencil offsets), so the
    effective bandwidths these models give exceed the HBM peak."""
    def nnz(nx, ny, nz):
        return (3 * nx - 2) * (3 * ny - 2) * (3 * nz - 2)
    lv = [(dims[0] >> l, dims[1] >> l, dims[2] >> l) for l in range(levels)]
    n = [a * b * c for a, b, c in lv]
    z = [nnz(*d) for d in lv]
    flops = 12 * n[0] + 2 * z[0] + sum(10 * z[l] for l in range(levels - 1)) + 4 * z[-1]
    b64 = 12 * z[0] + 16 * n[0] + 112 * n[0]
    b32 = b64
    for l in range(levels):
        sym64 = 24 * z[l] + 48 * n[l]
        sym32 = 12 * z[l] + (32 if l == 0 else 24) * n[l]
        if l < levels - 1:
            b64 += 2 * sym64 + 12 * z[l] + 16 * n[l] + 40 * n[l + 1]
            b32 += 2 * sym32 + 6 * z[l] + 8 * n[l] + 20 * n[l + 1]
        else:
            b64 += sym64
            b32 += sym32
    return flops, b64, b32, n[0], z[0]


class Clocks:
    """Samples SM clocks and throttle reasons while the timed region runs."""

    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + SMI_FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self, device_index):
        if not self.proc:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9 or p[0] != str(device_index):
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def sum_over_ranks(values, dist=None, device=None):
    """Element-wise sum of a list of floats over all ranks (identity on one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.tolist()


def max_over_ranks(values, dist=None, device=None):
    """Element-wise max of a list of floats over all ranks (identity on one rank).
    Every rank must call it with the same number of values."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


# The reference's own CG_ref (natural row order, src/CG_ref.cpp with
# src/ComputeSYMGS_ref.cpp) on the bench's system b = A u, u ~ U(-1, 1) seed 1,
# x0 = 0: iterations to ||r||/||r0|| <= 1e-10, measured with oracle/_ref
# (the reference compiled from its sources) on cubic grids.
REF_NATURAL_ITERS = {32: 24, 64: 40, 128: 71, 256: 128}


def reference_iterations(n):
    """CG_ref's iteration count to 1e-10 on the n^3 bench system: measured up
    to 256^3; beyond, each doubling of the grid multiplies the count by the
    ratio of the last measured doubling (geometric extrapolation)."""
    known = {k: v for k, v in REF_NATURAL_ITERS.items() if v > 0}
    if n in known:
        return known[n], "measured"
    top = max(known)
    prev = top // 2
    it, size = float(known[top]), top
    ratio = known[top] / float(known[prev])
    while size < n:
        it *= ratio
        size *= 2
    return int(round(it)), ("extrapolated from %d (%d^3) and %d (%d^3): x%.3f per doubling"
                            % (known[prev], prev, known[top], top, ratio))


def cpu_reference_sample(dims, sample_n=256, sample_it=3):
    """CG_ref of the reference build (oracle/_ref) on a sample_n^3 problem of
    the same kind (b = A u): the per-iteration time of a bounded run, scaled
    to dims rows and to CG_ref's own iteration count on dims."""
    from oracle.oracle import RefProblem, Oracle
    if not RefProblem.available():
        return None
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    ref = RefProblem(sample_n, sample_n, sample_n)
    n = ref.rows(0)
    u = Oracle.uniform(SEED_U, n, -1.0, 1.0)
    b = ref.spmv(0, u)
    t0 = time.perf_counter()
    _, k, nr, nr0, _ = ref.cg(b, np.zeros(n), sample_it, 0.0)
    dt = time.perf_counter() - t0
    ref.close()
    per_it = dt / k
    scale = (dims[0] * dims[1] * dims[2]) / float(n)
    iters, basis = reference_iterations(dims[0]) if dims[0] == dims[1] == dims[2] else (0, "")
    value = per_it * scale * iters
    return {"value": value, "unit": "s", "cores": int(os.environ.get("OMP_NUM_THREADS", threads)),
            "kind": "reference",
            "sample": "reference CG_ref (oracle/_ref, -O3 OpenMP, serial SYMGS as in "
                      "src/ComputeSYMGS_ref.cpp) on %d^3 (b = A u), %d iterations in %.2f s = "
                      "%.3f s/iter, measured; scaled x%.0f rows to %dx%dx%d and x%d iterations "
                      "(CG_ref's own count to 1e-10, %s)"
                      % (sample_n, k, dt, per_it, scale, dims[0], dims[1], dims[2], iters, basis),
            "measured_s_per_iteration": per_it, "sample_grid": [sample_n] * 3,
            "extrapolation": {"rows_factor": scale, "iterations": iters, "iterations_basis": basis}}


def run_reference(args, dims):
    """--impl reference: the reference's CPU path on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    vals = []
    cb = None
    for _ in range(args.warmup):
        if cpu_reference_sample(dims, sample_n=args.ref_sample, sample_it=1) is None:
            break
    for _ in range(max(1, args.steps)):
        cb = cpu_reference_sample(dims, sample_n=args.ref_sample, sample_it=args.ref_sample_it)
        if cb is None:
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref/libhpcgref.so not built (needs the "
                                             "reference sources at build time)"}))
            return
        vals.append(cb["value"])
    v = statistics.mean(vals)
    out = {"metric": METRIC, "value": v, "unit": "s", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
           "data": "synthetic (HPCG-generated problem, b = A u)",
           "config": config(dims), "cpu_baseline": dict(cb, value=v),
           "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def config(dims, world=1, sharded=False):
    g = (dims[0], dims[1], dims[2] * world) if sharded else dims
    c = {"workload": "HPCG %dx%dx%d (b = A u, u~U(-1,1) seed 1, x0 = 0): mixed-precision "
                     "flexible PCG (FP32/BF16 V-cycle, FP64 outer) to FP64 rel. residual "
                     "1e-10, compared with plain FP64 PCG" % g,
         "grid": list(g), "levels": 4, "smoother": "8-colour symmetric Gauss-Seidel",
         "tolerance": TOL, "l2": "no flush: every step streams > 60 GB, far above the 126 MB L2"}
    if world > 1:
        c["parallelism"] = ("z-slabs over %d GPUs (%dx%dx%d per GPU), NCCL halo exchange and "
                            "sums" % ((world,) + tuple(dims)) if sharded else
                            "%d independent replicas" % world)
    return c


def run_kernels(args):
    """Each plain operator of the reference's API on its own (256^3 by default):
    CUDA-event time of every call on the library's stream, algorithmic bytes of
    the reference implementation's step (real nonzeros only: SpMV 12 nnz + 16 n,
    SYMGS 24 nnz + 48 n, dot 16 n, WAXPBY 24 n) and their ratio against the
    measured HBM copy bandwidth.  Before each timed call the stream writes a
    256 MB buffer (L2 is 126 MB), so every call starts cold, and the stream is
    busy while the host enqueues the call; the calls are blocking API calls, so
    the time of the short vector operators still includes the launch of the
    call and the copy of its result to the host.  The command for the
    per-kernel ncu DRAM captures."""
    import torch
    from hpcg_b200 import Problem
    g = args.grid
    dims = (g[0], g[0], g[0]) if len(g) == 1 else tuple(g)
    torch.cuda.set_device(0)
    P = Problem(*dims)
    P.generate("hpcg")
    P.build_mixed()
    n = P.rows()
    flops, b64, b32, n0, nnz = model(dims)
    u = P.fill_uniform(SEED_U, -1.0, 1.0)
    v = P.fill_uniform(SEED_U + 1, 0.0, 1.0)
    x = P.fill_uniform(SEED_U + 2, 0.0, 1.0)
    y = torch.empty_like(u)
    u32 = u.float()
    ops = {
        "spmv": (lambda: P.spmv(u, y=y), 12 * nnz + 16 * n),
        "spmv_stencil": (lambda: P.spmv(u, y=y, stencil_cols=True), 8 * nnz + 16 * n),
        "symgs": (lambda: P.symgs(v, x), 24 * nnz + 48 * n),
        "dot": (lambda: P.dot(u, v), 16 * n),
        "waxpby": (lambda: P.waxpby(0.7, u, -1.3, v, w=y), 24 * n),
        "spmv_bf16": (lambda: P.spmv_mixed(u32), 2 * nnz + 8 * n),
    }
    peak, peak_kind = peaks()
    out = {"workload": "kernels", "grid": list(dims), "unit": "GB/s", "peak_gbs": peak,
           "peak_kind": peak_kind, "steps": args.steps, "warmup": args.warmup, "ops": {}}
    s = P.stream
    flush = torch.empty(32 << 20, dtype=torch.float64, device="cuda")
    for name, (f, nbytes) in ops.items():
        for _ in range(args.warmup):
            f()
        ts = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                flush.fill_(0.0)
            e0.record(s)
            f()
            e1.record(s)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        t = statistics.mean(ts)
        out["ops"][name] = {"ms": t * 1e3, "algorithmic_bytes": nbytes,
                            "achieved_gbs": nbytes / t / 1e9, "frac": nbytes / t / 1e9 / peak}
    print(json.dumps(out))
    P.close()


def run_varcoef(args):
    """Differentiable-solve workloads (no reference counterpart):
    (3) 128^3, a_ij = -exp(0.5 z) (seed 2), b ~ U(0,1), x_target ~ N(0,1) (seed 3),
        FP64 forward + adjoint to 1e-12, gradient vs central finite differences on 16
        edge-symmetric directions (seed 4);
    (4) 512x512x256, log-normal sigma = 1 (seed 5), b, x_target seed 6: mixed forward +
        adjoint to 1e-10, wall time, gradient error vs the FP64 adjoint."""
    import torch
    from hpcg_b200 import solve, symmetric_direction, varcoef_problem
    torch.cuda.set_device(0)
    out = {"workload": "varcoef", "unit": "s"}

    def loss(x, xt):
        return 0.5 * torch.sum((x - xt) ** 2)

    # ---- config 3: FD check
    g3 = args.grid3
    P, vals = varcoef_problem(g3, g3, g3, seed=2, sigma=0.5)
    n = P.rows()
    b = P.fill_uniform(3, 0.0, 1.0)
    xt = P.fill_normal(3, offset=n)
    v = vals.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    x = solve(v, bb, P, tol=1e-12)
    loss(x, xt).backward()
    xs = x.detach()
    gen = torch.Generator(device="cuda").manual_seed(4)
    errs = []
    for _ in range(16):
        Dv = symmetric_direction(P, gen) * vals.abs()
        Db = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
        h, dl = 1e-5, []
        for sgn in (1.0, -1.0):
            P.set_values((vals + sgn * h * Dv).reshape(-1), level=0, recoarsen=True)
            xp = xs.clone()
            P.cg(b + sgn * h * Db, xp, 2000, 1e-11)
            d = xp - xs
            dl.append(torch.sum(d * (xs - xt + 0.5 * d)).item())
        fd = (dl[0] - dl[1]) / (2 * h)
        an = (torch.sum(v.grad * Dv) + torch.sum(bb.grad * Db)).item()
        errs.append(abs(fd - an) / abs(an))
    out["config3"] = {"grid": [g3] * 3, "fd_rel_err_max": max(errs), "directions": 16,
                      "tolerance": 1e-12}
    P.close()
    del P, vals, v, bb, x, xs
    torch.cuda.empty_cache()
    # ---- config 4: mixed forward + adjoint, timed; FP64 adjoint for the error
    dims = tuple(args.grid4)
    P, vals = varcoef_problem(*dims, seed=5, sigma=1.0)
    P.build_mixed()
    n = P.rows()
    b = P.fill_uniform(6, 0.0, 1.0)
    xt = P.fill_normal(6, offset=n)
    res = {}
    for mixed in (True, False, True):       # first pass warms up, the last one is timed
        v = vals.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x = solve(v, bb, P, tol=1e-10, mixed=mixed)
        loss(x, xt).backward()
        torch.cuda.synchronize()
        res[mixed] = (time.perf_counter() - t0, v.grad, bb.grad)
        del v, bb, x
    t_mixed, gv_m, gb_m = res[True]
    t_fp64, gv_d, gb_d = res[False]
    out["config4"] = {
        "grid": list(dims), "fwd_bwd_s_mixed": t_mixed, "fwd_bwd_s_fp64": t_fp64,
        "speedup": t_fp64 / t_mixed,
        "grad_vals_rel_err_vs_fp64": (torch.linalg.norm(gv_m - gv_d) / torch.linalg.norm(gv_d)).item(),
        "grad_b_rel_err_vs_fp64": (torch.linalg.norm(gb_m - gb_d) / torch.linalg.norm(gb_d)).item(),
        "tolerance": 1e-10}
    print(json.dumps(out))


def run_slabs(args):
    """Iterations to 1e-10 of the sharded solver against the number of z-slabs
    (the reference's 1 x 1 x N process grid: SYMGS is block Jacobi across
    slabs, src/ComputeSYMGS_ref.cpp:56, so the count depends on N).  One
    global grid, split into N = 1, 2, 4, 8 slabs run as an in-process group on
    one GPU (hpcgx_group_cg: halo planes as device copies, sums in rank order)
    -- the algorithm of N GPUs, on one.  The system is the bench's b = A u,
    u ~ U(-1, 1) seed 1, x0 = 0, both solvers."""
    import torch
    from hpcg_b200 import Group, Problem
    from hpcg_b200._lib import CG_MG, CG_MIXED
    g = args.grid
    dims = (g[0], g[0], g[0]) if len(g) == 1 else tuple(g)
    torch.cuda.set_device(0)
    full = Problem(*dims)
    full.generate("hpcg")
    full.build_mixed()
    u = full.fill_uniform(SEED_U, -1.0, 1.0)
    b = full.spmv(u)
    out = {"workload": "slabs", "grid": list(dims), "tolerance": TOL,
           "system": "b = A u, u ~ U(-1,1) seed 1, x0 = 0", "slabs": {}}
    x = torch.zeros_like(b)
    row = {}
    for name, f in (("fp64", full.cg), ("mixed", full.cg_mixed)):
        x.zero_()
        k, nr, nr0 = f(b, x, MAX_IT, TOL)
        row[name] = k
    out["slabs"]["1"] = dict(row, solver="one-GPU graph solver")
    full.close()
    del full
    torch.cuda.empty_cache()
    for N in (2, 4, 8):
        if dims[2] % (N * 8):
            continue
        nz = dims[2] // N
        ranks = [Problem(dims[0], dims[1], nz, nranks=N, rank=r) for r in range(N)]
        for p in ranks:
            p.generate("hpcg")
            p.build_mixed()
        grp = Group(ranks)
        bs = [c.contiguous() for c in torch.split(b, b.numel() // N)]
        row = {}
        for name, mode in (("fp64", CG_MG), ("mixed", CG_MIXED)):
            xs = [torch.zeros_like(c) for c in bs]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            k, nr, nr0 = grp.cg(bs, xs, MAX_IT, TOL, mode=mode)
            torch.cuda.synchronize()
            row[name] = k
            row[name + "_rel_residual"] = nr / nr0
        out["slabs"][str(N)] = dict(row, solver="in-process group of %d slabs of %dx%dx%d"
                                    % (N, dims[0], dims[1], nz))
        grp.close()
        for p in ranks:
            p.close()
        torch.cuda.empty_cache()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hpcgx", choices=["hpcgx", "reference"])
    ap.add_argument("--grid", type=int, nargs="+", default=[512])
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N: N independent systems instead of one system sharded "
                         "into N z-slabs")
    ap.add_argument("--sharded", action="store_true",
                    help="the sharded step-by-step solver with an NCCL communicator even on one GPU")
    ap.add_argument("--clocks-csv", default="",
                    help="keep the nvidia-smi clock samples here (%%d = rank)")
    ap.add_argument("--ref-sample", type=int, default=256,
                    help="grid (n^3) of the reference's timed CPU sample")
    ap.add_argument("--ref-sample-it", type=int, default=3,
                    help="CG_ref iterations timed per sample")
    ap.add_argument("--workload", default="pcg", choices=["pcg", "varcoef", "kernels", "slabs"],
                    help="pcg: the headline metric; varcoef: the differentiable-solve checks; "
                         "kernels: each plain operator on its own (give --grid 256); slabs: "
                         "iterations against the number of z-slabs (give --grid 256)")
    ap.add_argument("--grid3", type=int, default=128)
    ap.add_argument("--grid4", type=int, nargs=3, default=[512, 512, 256])
    args = ap.parse_args()
    if args.workload == "varcoef":
        run_varcoef(args)
        return
    if args.workload == "kernels":
        run_kernels(args)
        return
    if args.workload == "slabs":
        run_slabs(args)
        return
    g = args.grid
    dims = (g[0], g[0], g[0]) if len(g) == 1 else tuple(g)

    if args.impl == "reference":
        run_reference(args, dims)
        return

    import torch
    # NCCL writes its log (a version line when NCCL_DEBUG is set) to stdout by
    # default; this process prints exactly one JSON line there
    os.environ.setdefault("NCCL_DEBUG_FILE",
                          os.path.join(tempfile.gettempdir(), "hpcgx_bench_nccl.%h.%p.log"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    # no legitimate wait between two collectives of this run lasts more than a
    # few seconds (one problem generation, one solve's per-iteration sums), so
    # a rank that waits two minutes on its peers has lost one: end with an error
    os.environ.setdefault("HPCGX_WAIT_TIMEOUT_S", "120")
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)

    from hpcg_b200 import Problem, nccl_unique_id
    from hpcg_b200._lib import CG_MG, CG_MIXED, PROBE_GS_FINE, PROBE_GS_FINE_BWD, PROBE_SPMV_FINE

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # N > 1: one nx x ny x (nz N) system, z-slab `rank` on this GPU (weak
    # scaling: every GPU holds one dims-sized slab), halos and sums over NCCL
    sharded = (world > 1 and not args.replicas) or args.sharded
    if sharded:
        P = Problem(*dims, device=dev, nranks=world, rank=rank)
    else:
        P = Problem(*dims, device=dev)
    P.generate("hpcg")
    P.build_mixed()
    if sharded:
        uid = [nccl_unique_id() if rank == 0 else None]
        if dist:
            dist.broadcast_object_list(uid, src=0, device=torch.device("cuda", dev))
        P.attach_nccl(uid[0])

    def gnorm(v):
        """2-norm of the global vector whose slab this rank holds."""
        s = float(torch.dot(v, v))
        return sum_over_ranks([s], dist if (sharded and dist) else None, f"cuda:{dev}")[0] ** 0.5
    n = P.rows()
    u = P.fill_uniform(SEED_U, -1.0, 1.0)
    b = P.spmv(u)
    x = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    stream = P.stream

    def solve(mixed):
        x.zero_()
        f = P.cg_mixed if mixed else P.cg
        return f(b, x, MAX_IT, TOL)

    # ---------------- warm-up (untimed); the probe is armed first so that the
    # solver's CUDA graph (with its event nodes) is captured here, not in the
    # timed region
    P.set_probe(PROBE_GS_FINE | PROBE_GS_FINE_BWD | PROBE_SPMV_FINE)
    for _ in range(args.warmup):
        solve(True)
    # ---------------- timed mixed solves
    for kind in (PROBE_GS_FINE, PROBE_GS_FINE_BWD, PROBE_SPMV_FINE):
        P.probe_read(kind, reset=True)
    barrier()
    l0 = P.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    iters_mixed = []
    clk = Clocks(args.clocks_csv % rank if args.clocks_csv else
                 os.path.join(tempfile.gettempdir(), "hpcgx_bench_clocks_rank%d.csv" % rank))
    with clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                ev[i][0].record(stream)
            k, nr, nr0 = solve(True)
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
            iters_mixed.append(k)
        barrier()
        wall = time.perf_counter() - t0
    launches = P.launch_count() - l0
    times = [a.elapsed_time(b_) * 1e-3 for a, b_ in ev]
    probes = {k: P.probe_read(k, reset=True)
              for k in (PROBE_GS_FINE, PROBE_GS_FINE_BWD, PROBE_SPMV_FINE)}
    P.set_probe(0)
    t_mixed = statistics.mean(times)
    relres_mixed = nr / nr0
    x_mixed = x.clone()
    true_mixed = gnorm(b - P.spmv(x_mixed)) / gnorm(b)

    # ---------------- FP64 comparison
    solve(False)
    t64 = []
    for _ in range(max(1, args.fp64_steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        k64, nr64, nr064 = solve(False)
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        t64.append(e0.elapsed_time(e1) * 1e-3)
    t_fp64 = statistics.mean(t64)
    # bytes of one iteration as this implementation moves them (one-GPU
    # solver; read while each solver's iteration graph is current)
    ib = {}
    if not sharded:
        ib = {"mixed": P.iteration_bytes(CG_MIXED), "fp64": P.iteration_bytes(CG_MG)}
    x64 = x.clone()
    true_fp64 = gnorm(b - P.spmv(x64)) / gnorm(b)
    x_diff = gnorm(x_mixed - x64) / gnorm(x64)
    err_u = gnorm(x_mixed - u) / gnorm(u)

    # ---------------- FP64 with the mixed solver's column derivation: the FP64
    # solve that differs from the mixed one in precision only (every column
    # from the stencil offsets, no int32 column reads)
    P.set_stencil_columns(True)
    solve(False)
    t64s = []
    for _ in range(max(1, args.fp64_steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        k64s, nr64s, nr064s = solve(False)
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        t64s.append(e0.elapsed_time(e1) * 1e-3)
    t_fp64s = statistics.mean(t64s)
    x64s_diff = gnorm(x - x64) / gnorm(x64)
    if not sharded:
        ib["fp64_stencil_cols"] = P.iteration_bytes(CG_MG)
    P.set_stencil_columns(False)

    # ---------------- end to end through the C ABI from pinned host buffers:
    # b copied in and x copied out inside each timed solve
    bh = b.cpu().pin_memory()
    xh = torch.zeros(n, dtype=torch.float64).pin_memory()
    P.cg_host(bh.numpy(), xh.numpy(), MAX_IT, TOL, mixed=True)   # untimed warm-up
    te2e = []
    for _ in range(args.steps):
        xh.zero_()
        barrier()
        te = time.perf_counter()
        ke, nre, nr0e = P.cg_host(bh.numpy(), xh.numpy(), MAX_IT, TOL, mixed=True)
        torch.cuda.synchronize()
        te2e.append(time.perf_counter() - te)
    t_e2e = statistics.mean(te2e)

    # ---------------- max over ranks
    t_mixed, t_fp64, t_fp64s, t_e2e = max_over_ranks([t_mixed, t_fp64, t_fp64s, t_e2e], dist,
                                                     f"cuda:{dev}")

    flops, b64, b32, n0, z0 = model(dims)
    peak, peak_kind = peaks()
    # whole job: every rank does one slab's (or one replica's) work per iteration
    gf_mixed = world * flops * iters_mixed[-1] / t_mixed / 1e9
    gf_fp64 = world * flops * k64 / t_fp64 / 1e9
    ref_mixed = world * b32 * iters_mixed[-1] / t_mixed / 1e9
    ref_fp64 = world * b64 * k64 / t_fp64 / 1e9

    def whole_iteration(kind, iters, t):
        if kind not in ib:
            return None
        ach = world * ib[kind] * iters / t / 1e9
        return {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "bytes_per_iteration": ib[kind], "iterations": iters, "time_s": t,
                "peak_kind": peak_kind}
    traffic = {}
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic_%d.json" % dims[0])
    if os.path.exists(tpath) and dims[0] == dims[1] == dims[2]:
        try:
            traffic = json.load(open(tpath))
        except Exception:
            traffic = {}

    def roofline(kind, name):
        ms, cnt, by = probes[kind]
        ach = by / (ms * 1e-3) / 1e9 if ms > 0 else None
        tr = traffic.get(name, {}).get("dram_bytes_per_launch") if traffic else None
        return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": (ach / peak) if ach else None, "traffic": tr,
                "algorithmic_bytes_per_launch": (by / cnt) if cnt else None,
                "launches": cnt, "mean_launch_ms": (ms / cnt) if cnt else None,
                "peak_kind": peak_kind}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu and world == 1:   # the CPU sample is taken at N = 1 only
        try:
            cpu = cpu_reference_sample(dims)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"unavailable": str(e)}
    clocks = clk.summary(dev)
    out = {
        "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64 outer / fp32+bf16 V-cycle",
        "data": "synthetic (HPCG-generated problem on the device, b = A u)",
        "config": config(dims, world, sharded),
        "iterations": {"mixed": iters_mixed[-1], "fp64": k64},
        "fp64_time_s": t_fp64,
        "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
        "fp64_stencil_cols_time_s": t_fp64s,
        "speedup_mixed_vs_fp64_stencil_cols": t_fp64s / t_mixed,
        "fp64_stencil_cols": {"iterations": k64s, "x_rel_diff_vs_fp64": x64s_diff,
                              "note": "FP64 PCG with every column derived from the stencil "
                                      "offsets, as the mixed solver does: the mixed-vs-FP64 "
                                      "ratio from precision alone"},
        "fp64_rel_residual": {"mixed_recursive": relres_mixed, "mixed_true": true_mixed,
                              "fp64_true": true_fp64},
        "x_rel_diff_vs_fp64": x_diff, "x_rel_err_vs_u": err_u,
        "gflops": {"mixed": gf_mixed, "fp64": gf_fp64, "model": "src/ReportResults.cpp:81-97"},
        "roofline_iteration": {
            "mixed": whole_iteration("mixed", iters_mixed[-1], t_mixed),
            "fp64": whole_iteration("fp64", k64, t_fp64),
            "fp64_stencil_cols": whole_iteration("fp64_stencil_cols", k64s, t_fp64s),
            "model": "this implementation's algorithmic bytes per CG iteration "
                     "(hpcgx_iteration_bytes: every launch of the iteration, real nonzeros, each "
                     "vector element once per launch) x iterations / solve time"},
        "reference_model_gbs": {"mixed": ref_mixed, "fp64": ref_fp64,
                                "model": "bytes per iteration of the reference implementation's "
                                         "steps (SpMV 12 nnz + 16 n, SYMGS 24 nnz + 48 n, R+P "
                                         "40 n_c, CG vectors 112 n; mixed V-cycle 6 B/nnz, FP32 "
                                         "vectors) / time: work this design does not do, so it "
                                         "exceeds the HBM peak; for comparison with other HPCG "
                                         "implementations only"},
        "roofline": roofline(PROBE_SPMV_FINE, "k_spmv<double,double,1,1>"),
        "roofline_gs_bwd": roofline(PROBE_GS_FINE_BWD, "k_gs_class<0,1,-1,bf16,f32,f32>"),
        "roofline_gs_fine_all_modes": roofline(PROBE_GS_FINE, "k_gs_class finest level, all modes"),
        "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": world * 2 * n * 8,
                "d2h_bytes_per_step": world * n * 8, "steps": args.steps},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "wall_s": wall,
    }
    print(json.dumps(out))
    P.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
