"""Python host API over libhpcgx: HPCG's operators on torch CUDA tensors.

``Problem`` mirrors the reference's replaceable operator set
(src/ComputeSPMV.hpp, ComputeSYMGS.hpp, ComputeMG.hpp, ComputeDotProduct.hpp,
ComputeWAXPBY.hpp, ComputeResidual.hpp, CG.hpp, OptimizeProblem.hpp) with the
same argument meaning and the same 0/non-zero status convention, turned into
Python exceptions (``HPCGXError``).  Vectors are float64 (float32 for the
mixed-precision V-cycle) CUDA tensors in natural row order.

All library work runs on one torch stream owned by the problem; every call
first makes that stream wait for the caller's current stream, and returns
after the library has synchronised, so results are ready when a method
returns.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

STENCIL = 27


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data_as(C.c_void_p)
    return C.c_void_p(t.data_ptr())


class Problem:
    """One nx*ny*nz HPCG problem with ``levels`` multigrid levels on a GPU.

    With ``nranks`` > 1 it is z-slab ``rank`` of an nx*ny*(nz*nranks) problem
    (the reference's 1 x 1 x nranks process grid): attach a communicator with
    :meth:`attach_nccl` (one process per GPU) or tie all slabs of one process
    into a :class:`Group`.
    """

    def __init__(self, nx, ny, nz, levels=4, device=0, nranks=1, rank=0):
        if not torch.cuda.is_available():
            raise RuntimeError("hpcg_b200 needs a CUDA device")
        self.dims = (nx, ny, nz)
        self.levels = levels
        self.nranks, self.rank = nranks, rank
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        check(lib().hpcgx_create_slab(device, nx, ny, nz, levels, nranks, rank, C.byref(h)))
        self.h = h
        self.stream = torch.cuda.Stream(device=self.device)
        check(lib().hpcgx_set_stream(self.h, C.c_void_p(self.stream.cuda_stream)))
        self.values_version = 0     # bumped whenever matrix values change

    @classmethod
    def general(cls, levels=4, device=0):
        """A general-pattern problem (hpcgx_create_general): each level is
        loaded as given with :meth:`load_level_general` -- any sparsity
        pattern, the multicolouring computed from the matrix graph."""
        if not torch.cuda.is_available():
            raise RuntimeError("hpcg_b200 needs a CUDA device")
        self = cls.__new__(cls)
        self.dims = None
        self.levels = levels
        self.nranks, self.rank = 1, 0
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        check(lib().hpcgx_create_general(device, levels, C.byref(h)))
        self.h = h
        self.stream = torch.cuda.Stream(device=self.device)
        check(lib().hpcgx_set_stream(self.h, C.c_void_p(self.stream.cuda_stream)))
        self.values_version = 0
        return self

    def load_level_general(self, level, nnz, cols, vals, f2c=None):
        """Rows of any pattern: row i holds nnz[i] entries in cols[i, :nnz[i]] /
        vals[i, :nnz[i]] (2-D arrays, one row per matrix row, entries in the
        order the row sums them); f2c: the injection to the next level."""
        nnz = np.ascontiguousarray(nnz, np.uint8)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        n, w = cols.shape
        cptr = (C.c_void_p * n)(*(cols.ctypes.data + 4 * w * np.arange(n)).tolist())
        vptr = (C.c_void_p * n)(*(vals.ctypes.data + 8 * w * np.arange(n)).tolist())
        fc = None if f2c is None else np.ascontiguousarray(f2c, np.int32)
        check(lib().hpcgx_load_level_general(self.h, level, n, _ptr(nnz), cptr, vptr, _ptr(fc),
                                             0 if fc is None else fc.size))
        self.values_version += 1

    def colours(self, level=0):
        return int(lib().hpcgx_colours(self.h, level))

    # ----------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "h", None):
            lib().hpcgx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _pre(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))

    def rows(self, level=0):
        return int(lib().hpcgx_rows(self.h, level))

    def attach_nccl(self, unique_id: bytes):
        """Joins the NCCL communicator of the problem's ranks (collective); the
        operators and CG then exchange halos and sum reductions over NCCL."""
        buf = C.create_string_buffer(bytes(unique_id), _lib.NCCL_ID_BYTES)
        check(lib().hpcgx_attach_nccl(self.h, buf, _lib.NCCL_ID_BYTES))

    def attach_comm(self, halo, sum_):
        """A caller's own transport (hpcgx_attach_comm): ``halo(send_lo, recv_lo,
        send_hi, recv_hi, count, esize, stream)`` and ``sum_(buf, count, stream)``
        take device pointers (int, 0 = no neighbour) and the library's stream
        handle, and return nothing; an exception becomes HPCGX_ECOMM."""
        import traceback

        def _halo(ctx, slo, rlo, shi, rhi, count, esize, stream):
            try:
                halo(slo or 0, rlo or 0, shi or 0, rhi or 0, int(count), int(esize), stream or 0)
                return 0
            except Exception:
                traceback.print_exc()
                return 1

        def _sum(ctx, buf, count, stream):
            try:
                sum_(buf or 0, int(count), stream or 0)
                return 0
            except Exception:
                traceback.print_exc()
                return 1

        self._comm_fns = (_lib.HALO_FN(_halo), _lib.SUM_FN(_sum))   # kept alive with the problem
        check(lib().hpcgx_attach_comm(self.h, self._comm_fns[0], self._comm_fns[1], None))

    def attach_torch_distributed(self, group=None):
        """Exchanges halos and sums over torch.distributed (any backend; gloo
        moves them through host memory), rank = this problem's slab."""
        import torch.distributed as dist
        dev = self.device

        def view(ptr, count, esize):
            typestr = "<f8" if esize == 8 else "<f4"
            return torch.as_tensor(_DeviceArray(ptr, count, typestr), device=dev)

        def on_host(t):
            return t.cpu() if dist.get_backend(group) == "gloo" else t

        def halo(slo, rlo, shi, rhi, count, esize, stream):
            torch.cuda.ExternalStream(stream, device=dev).synchronize()
            reqs, into = [], []
            for send, recv, peer in ((slo, rlo, self.rank - 1), (shi, rhi, self.rank + 1)):
                if not send:
                    continue
                out = on_host(view(send, count, esize).clone())
                got = torch.empty_like(out)
                reqs += [dist.isend(out, peer, group=group), dist.irecv(got, peer, group=group)]
                into.append((recv, got))
            for q in reqs:
                q.wait()
            for recv, got in into:
                view(recv, count, esize).copy_(got)
            torch.cuda.synchronize(dev)

        def sum_(buf, count, stream):
            torch.cuda.ExternalStream(stream, device=dev).synchronize()
            t = on_host(view(buf, count, 8).clone())
            dist.all_reduce(t, group=group)
            view(buf, count, 8).copy_(t)
            torch.cuda.synchronize(dev)

        self.attach_comm(halo, sum_)

    def level_dims(self, level=0):
        if self.dims is None:
            raise ValueError("a general-pattern problem has no grid")
        nx, ny, nz = self.dims
        return nx >> level, ny >> level, nz >> level

    def empty(self, level=0, dtype=torch.float64):
        return torch.empty(self.rows(level), dtype=dtype, device=self.device)

    def zeros(self, level=0, dtype=torch.float64):
        return torch.zeros(self.rows(level), dtype=dtype, device=self.device)

    # ----------------------------------------------------------- set-up
    def generate(self, kind="hpcg", seed=0, sigma=0.0):
        code = {"hpcg": _lib.GEN_HPCG, "varcoef": _lib.GEN_VARCOEF}[kind]
        check(lib().hpcgx_generate(self.h, code, seed, float(sigma)))
        self.values_version += 1
        return self

    def load_level(self, level, nnz, cols, vals):
        """Host matrix in the reference's contiguous 27-slot row layout."""
        nnz = np.ascontiguousarray(nnz, np.uint8)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        check(lib().hpcgx_load_level(self.h, level, _ptr(nnz), _ptr(cols), _ptr(vals)))
        self.values_version += 1

    def check_f2c(self, level, f2c):
        f2c = np.ascontiguousarray(f2c, np.int32)
        check(lib().hpcgx_check_f2c(self.h, level, _ptr(f2c), f2c.size))

    def build_mixed(self):
        check(lib().hpcgx_build_mixed(self.h))

    def set_stencil_columns(self, on=True):
        """FP64 operators derive their columns from the stencil offsets (the
        mixed solver always does); same results, no int32 column reads."""
        check(lib().hpcgx_set_stencil_columns(self.h, int(bool(on))))

    def set_diagonal(self, level, diag):
        d = np.ascontiguousarray(diag, np.float64)
        check(lib().hpcgx_set_diagonal_host(self.h, level, _ptr(d)))
        self.values_version += 1

    def get_diagonal(self, level=0):
        d = np.zeros(self.rows(level))
        check(lib().hpcgx_get_diagonal_host(self.h, level, _ptr(d)))
        return d

    def set_values(self, vals27, level=0, recoarsen=False):
        self._pre()
        v = vals27.contiguous()
        check(lib().hpcgx_set_values(self.h, level, _ptr(v), int(recoarsen)))
        self.values_version += 1

    def get_values(self, level=0):
        self._pre()
        n = self.rows(level)
        v = torch.empty(n * STENCIL, dtype=torch.float64, device=self.device)
        c = torch.empty(n * STENCIL, dtype=torch.int32, device=self.device)
        check(lib().hpcgx_get_values(self.h, level, _ptr(v), _ptr(c)))
        return v.view(n, STENCIL), c.view(n, STENCIL)

    def memory_bytes(self):
        b = C.c_double()
        check(lib().hpcgx_memory_bytes(self.h, C.byref(b)))
        return b.value

    # ----------------------------------------------------------- operators
    def spmv(self, x, level=0, y=None, stencil_cols=False):
        """y = A x; stencil_cols derives the columns from the stencil offsets."""
        self._pre()
        y = self.empty(level) if y is None else y
        f = lib().hpcgx_spmv_stencil if stencil_cols else lib().hpcgx_spmv
        check(f(self.h, level, _ptr(x), _ptr(y)))
        return y

    def symgs(self, r, x, level=0):
        """One symmetric Gauss-Seidel sweep, x updated in place."""
        self._pre()
        check(lib().hpcgx_symgs(self.h, level, _ptr(r), _ptr(x)))
        return x

    def mg(self, r, x=None):
        self._pre()
        x = self.empty(0) if x is None else x
        check(lib().hpcgx_mg(self.h, _ptr(r), _ptr(x)))
        return x

    def restriction(self, level, rf, Axf):
        self._pre()
        rc = self.empty(level + 1)
        check(lib().hpcgx_restriction(self.h, level, _ptr(rf), _ptr(Axf), _ptr(rc)))
        return rc

    def prolongation(self, level, xc, xf):
        self._pre()
        check(lib().hpcgx_prolongation(self.h, level, _ptr(xc), _ptr(xf)))
        return xf

    def dot(self, x, y):
        self._pre()
        out = C.c_double()
        check(lib().hpcgx_dot(self.h, x.numel(), _ptr(x), _ptr(y), C.byref(out)))
        return out.value

    def waxpby(self, alpha, x, beta, y, w=None):
        self._pre()
        w = torch.empty_like(x) if w is None else w
        check(lib().hpcgx_waxpby(self.h, x.numel(), float(alpha), _ptr(x), float(beta), _ptr(y),
                                 _ptr(w)))
        return w

    def residual(self, v1, v2):
        self._pre()
        out = C.c_double()
        check(lib().hpcgx_residual(self.h, v1.numel(), _ptr(v1), _ptr(v2), C.byref(out)))
        return out.value

    # mixed precision --------------------------------------------------
    def spmv_mixed(self, x32, level=0):
        self._pre()
        y = self.empty(level, torch.float32)
        check(lib().hpcgx_spmv_mixed(self.h, level, _ptr(x32), _ptr(y)))
        return y

    def symgs_mixed(self, r, x32, level=0):
        self._pre()
        r64 = r if r.dtype == torch.float64 else None
        r32 = r if r.dtype == torch.float32 else None
        check(lib().hpcgx_symgs_mixed(self.h, level, _ptr(r64), _ptr(r32), _ptr(x32)))
        return x32

    def mg_mixed(self, r, x32=None):
        self._pre()
        x32 = self.empty(0, torch.float32) if x32 is None else x32
        check(lib().hpcgx_mg_mixed(self.h, _ptr(r), _ptr(x32)))
        return x32

    # ----------------------------------------------------------- solvers
    def cg(self, b, x, max_iter, tol, precond=True, times=None):
        """Returns (niters, normr, normr0); x is updated in place."""
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        tp = _ptr(times) if times is not None else None
        check(lib().hpcgx_cg(self.h, _ptr(b), _ptr(x), int(max_iter), float(tol), int(precond),
                             C.byref(it), C.byref(nr), C.byref(nr0), tp))
        return it.value, nr.value, nr0.value

    def cg_mixed(self, b, x, max_iter, tol, times=None):
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        tp = _ptr(times) if times is not None else None
        check(lib().hpcgx_cg_mixed(self.h, _ptr(b), _ptr(x), int(max_iter), float(tol),
                                   C.byref(it), C.byref(nr), C.byref(nr0), tp))
        return it.value, nr.value, nr0.value

    def cg_host(self, b_host, x_host, max_iter, tol, mixed=False, precond=True, times=None):
        """Solve from host buffers (numpy or pinned CPU tensors); x_host updated."""
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        tp = _ptr(times) if times is not None else None
        mode = _lib.CG_MIXED if mixed else (_lib.CG_MG if precond else _lib.CG_PLAIN)
        check(lib().hpcgx_cg_host(self.h, mode, _ptr(b_host), _ptr(x_host), int(max_iter),
                                  float(tol), C.byref(it), C.byref(nr), C.byref(nr0), tp))
        return it.value, nr.value, nr0.value

    # ----------------------------------------------------------- adjoint
    def adjoint_grad(self, lam, x):
        self._pre()
        n = self.rows(0)
        g = torch.empty(n * STENCIL, dtype=torch.float64, device=self.device)
        check(lib().hpcgx_adjoint_grad(self.h, _ptr(lam), _ptr(x), _ptr(g)))
        return g.view(n, STENCIL)

    # ----------------------------------------------------------- inputs
    def fill_uniform(self, seed, lo=0.0, hi=1.0, n=None):
        self._pre()
        n = self.rows(0) if n is None else n
        v = torch.empty(n, dtype=torch.float64, device=self.device)
        check(lib().hpcgx_fill_uniform(self.h, n, seed, float(lo), float(hi), _ptr(v)))
        return v

    def fill_normal(self, seed, offset=0, n=None):
        self._pre()
        n = self.rows(0) if n is None else n
        v = torch.empty(n, dtype=torch.float64, device=self.device)
        check(lib().hpcgx_fill_normal(self.h, n, seed, offset, _ptr(v)))
        return v

    # ----------------------------------------------------------- measurement
    def set_probe(self, probe):
        check(lib().hpcgx_set_probe(self.h, int(probe)))

    def probe_read(self, kind=_lib.PROBE_GS_FINE, reset=True):
        """(summed device ms, launches, algorithmic bytes) of one probe kind."""
        ms, n, b = C.c_double(), C.c_int64(), C.c_double()
        check(lib().hpcgx_probe_read(self.h, int(kind), C.byref(ms), C.byref(n), C.byref(b),
                                     int(reset)))
        return ms.value, n.value, b.value

    def iteration_bytes(self, mode=_lib.CG_MIXED):
        """Algorithmic bytes of one CG iteration of ``mode`` (this
        implementation's byte model, summed over the iteration's launches);
        available after a solve of that mode."""
        out = C.c_double()
        check(lib().hpcgx_iteration_bytes(self.h, int(mode), C.byref(out)))
        return out.value

    def launch_count(self):
        return int(lib().hpcgx_launch_count(self.h))

    def synchronize(self):
        check(lib().hpcgx_synchronize(self.h))


def check_status() -> None:
    """Raises HPCGXError(ECHECK) if a kernel of the index-checked build
    (HPCGX_LIBRARY=checked) met an out-of-range index since the last call."""
    check(lib().hpcgx_check_status())


def nccl_unique_id() -> bytes:
    """A fresh NCCL unique id (rank 0 makes it; every rank attaches with it)."""
    buf = C.create_string_buffer(_lib.NCCL_ID_BYTES)
    check(lib().hpcgx_nccl_unique_id(buf, _lib.NCCL_ID_BYTES))
    return buf.raw


class _DeviceArray:
    """A device buffer owned by the library, seen by torch through the CUDA
    array interface."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _ptrs(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


class Group:
    """Every z-slab of a sharded problem in one process on one GPU.

    The slabs run in lockstep on the stream of slab 0: halo planes are copied
    between the slabs' vectors and reductions are summed in rank order, which
    is the multi-rank algorithm (block-Jacobi smoothing across slabs, sums over
    ranks) on a single device.  Vector arguments are lists with one tensor per
    rank.
    """

    def __init__(self, ranks):
        self.ranks = list(ranks)
        handles = (C.c_void_p * len(self.ranks))(*[p.h.value for p in self.ranks])
        g = C.c_void_p()
        check(lib().hpcgx_group_create(handles, len(self.ranks), C.byref(g)))
        self.g = g
        self.stream = self.ranks[0].stream

    def close(self):
        if getattr(self, "g", None):
            lib().hpcgx_group_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pre(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.ranks[0].device))

    def spmv(self, xs, level=0):
        self._pre()
        ys = [p.empty(level) for p in self.ranks]
        check(lib().hpcgx_group_spmv(self.g, level, _ptrs(xs), _ptrs(ys)))
        return ys

    def symgs(self, rs, xs, level=0):
        """One symmetric sweep per slab (block Jacobi across slabs), x in place."""
        self._pre()
        check(lib().hpcgx_group_symgs(self.g, level, _ptrs(rs), _ptrs(xs)))
        return xs

    def mg(self, rs):
        self._pre()
        xs = [p.empty(0) for p in self.ranks]
        check(lib().hpcgx_group_mg(self.g, _ptrs(rs), _ptrs(xs)))
        return xs

    def cg(self, bs, xs, max_iter, tol, mode=_lib.CG_MG):
        """CG over the slabs; xs updated in place; returns (iters, normr, normr0)."""
        self._pre()
        k, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        check(lib().hpcgx_group_cg(self.g, mode, _ptrs(bs), _ptrs(xs), max_iter, tol,
                                   C.byref(k), C.byref(nr), C.byref(nr0)))
        return k.value, nr.value, nr0.value
