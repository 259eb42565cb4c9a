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


F64 = (torch.float64,)
F32 = (torch.float32,)


def _dev(t, n, dtypes, device, name):
    """The device pointer of a vector argument, after the checks the C ABI
    cannot make on a raw pointer: a contiguous torch tensor of one of
    ``dtypes`` on the problem's device with at least ``n`` entries (the
    kernels read or write that many through the pointer).  A host array or a
    tensor of another device would be dereferenced by the GPU, and a short or
    strided one read past its end."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch tensor on {device}, got {type(t).__name__}")
    if t.device != device:
        raise ValueError(f"{name}: the tensor is on {t.device}, the problem on {device}")
    if t.dtype not in dtypes:
        raise TypeError(f"{name}: dtype {t.dtype}, expected " + " or ".join(map(str, dtypes)))
    if not t.is_contiguous():
        raise ValueError(f"{name}: the tensor is not contiguous")
    if t.numel() < n:
        raise ValueError(f"{name}: {t.numel()} entries, the operator uses {n}")
    return C.c_void_p(t.data_ptr())


def _host(a, n, name):
    """The pointer of a host float64 vector (numpy array or CPU tensor, used in
    place: outputs are written into it) of at least ``n`` entries."""
    if isinstance(a, torch.Tensor):
        if a.device.type != "cpu":
            raise ValueError(f"{name}: expected host memory, the tensor is on {a.device}")
        a = a.detach().numpy()
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{name}: expected a numpy array or CPU tensor, got {type(a).__name__}")
    if a.dtype != np.float64:
        raise TypeError(f"{name}: dtype {a.dtype}, expected float64")
    if not a.flags.c_contiguous:
        raise ValueError(f"{name}: the array is not contiguous")
    if a.size < n:
        raise ValueError(f"{name}: {a.size} entries, the operator uses {n}")
    return a.ctypes.data_as(C.c_void_p)


def _at_least(a, n, name):
    """Size check of a host input array (already converted to its C type)."""
    if a.size < n:
        raise ValueError(f"{name}: {a.size} entries, the level needs {n}")
    return a


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
        nnz = np.ascontiguousarray(nnz, np.uint8).reshape(-1)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        if cols.ndim != 2 or vals.shape != cols.shape:
            raise ValueError(f"cols {cols.shape} and vals {vals.shape}: expected two arrays "
                             "of the same (rows, width) shape")
        n, w = cols.shape
        if nnz.size != n:
            raise ValueError(f"nnz: {nnz.size} entries for {n} rows")
        if n and int(nnz.max()) > w:
            raise ValueError(f"nnz: a row holds {int(nnz.max())} entries, wider than the "
                             f"arrays ({w})")
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
        n = self.rows(level)
        nnz = _at_least(np.ascontiguousarray(nnz, np.uint8), n, "nnz")
        cols = _at_least(np.ascontiguousarray(cols, np.int32), STENCIL * n, "cols")
        vals = _at_least(np.ascontiguousarray(vals, np.float64), STENCIL * n, "vals")
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
        d = _at_least(np.ascontiguousarray(diag, np.float64), self.rows(level), "diag")
        check(lib().hpcgx_set_diagonal_host(self.h, level, _ptr(d)))
        self.values_version += 1

    def get_diagonal(self, level=0):
        d = np.zeros(self.rows(level))
        check(lib().hpcgx_get_diagonal_host(self.h, level, _ptr(d)))
        return d

    def set_values(self, vals27, level=0, recoarsen=False):
        self._pre()
        v = vals27.contiguous()
        check(lib().hpcgx_set_values(self.h, level,
                                     _dev(v, STENCIL * self.rows(level), F64, self.device,
                                          "vals27"), int(recoarsen)))
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
    def _v(self, t, level, name, dtypes=F64):
        return _dev(t, self.rows(level), dtypes, self.device, name)

    def spmv(self, x, level=0, y=None, stencil_cols=False):
        """y = A x; stencil_cols derives the columns from the stencil offsets."""
        self._pre()
        y = self.empty(level) if y is None else y
        f = lib().hpcgx_spmv_stencil if stencil_cols else lib().hpcgx_spmv
        check(f(self.h, level, self._v(x, level, "x"), self._v(y, level, "y")))
        return y

    def symgs(self, r, x, level=0):
        """One symmetric Gauss-Seidel sweep, x updated in place."""
        self._pre()
        check(lib().hpcgx_symgs(self.h, level, self._v(r, level, "r"), self._v(x, level, "x")))
        return x

    def mg(self, r, x=None):
        self._pre()
        x = self.empty(0) if x is None else x
        check(lib().hpcgx_mg(self.h, self._v(r, 0, "r"), self._v(x, 0, "x")))
        return x

    def restriction(self, level, rf, Axf):
        self._pre()
        rc = self.empty(level + 1)
        check(lib().hpcgx_restriction(self.h, level, self._v(rf, level, "rf"),
                                      self._v(Axf, level, "Axf"), _ptr(rc)))
        return rc

    def prolongation(self, level, xc, xf):
        self._pre()
        check(lib().hpcgx_prolongation(self.h, level, self._v(xc, level + 1, "xc"),
                                       self._v(xf, level, "xf")))
        return xf

    def _n(self, x, name="x"):
        """n of a length-n vector operation: all of x, on the problem's device."""
        return _dev(x, 0, F64, self.device, name), x.numel()

    def dot(self, x, y):
        self._pre()
        px, n = self._n(x)
        out = C.c_double()
        check(lib().hpcgx_dot(self.h, n, px, _dev(y, n, F64, self.device, "y"), C.byref(out)))
        return out.value

    def waxpby(self, alpha, x, beta, y, w=None):
        self._pre()
        px, n = self._n(x)
        w = torch.empty_like(x) if w is None else w
        check(lib().hpcgx_waxpby(self.h, n, float(alpha), px, float(beta),
                                 _dev(y, n, F64, self.device, "y"),
                                 _dev(w, n, F64, self.device, "w")))
        return w

    def residual(self, v1, v2):
        self._pre()
        p1, n = self._n(v1, "v1")
        out = C.c_double()
        check(lib().hpcgx_residual(self.h, n, p1, _dev(v2, n, F64, self.device, "v2"),
                                   C.byref(out)))
        return out.value

    # mixed precision --------------------------------------------------
    def spmv_mixed(self, x32, level=0):
        self._pre()
        y = self.empty(level, torch.float32)
        check(lib().hpcgx_spmv_mixed(self.h, level, self._v(x32, level, "x32", F32), _ptr(y)))
        return y

    def symgs_mixed(self, r, x32, level=0):
        """One FP32 sweep with BF16 values; r is float64 or float32."""
        self._pre()
        pr = self._v(r, level, "r", F64 + F32)
        r64, r32 = (pr, None) if r.dtype == torch.float64 else (None, pr)
        check(lib().hpcgx_symgs_mixed(self.h, level, r64, r32, self._v(x32, level, "x32", F32)))
        return x32

    def mg_mixed(self, r, x32=None):
        self._pre()
        x32 = self.empty(0, torch.float32) if x32 is None else x32
        check(lib().hpcgx_mg_mixed(self.h, self._v(r, 0, "r"), self._v(x32, 0, "x32", F32)))
        return x32

    # ----------------------------------------------------------- solvers
    def _times(self, times):
        """CG's host times array: the library adds to entries 0 (total), 2
        (vector operations), 3 (SpMV) and 5 (preconditioner), the slots of
        src/CG.cpp:133-141."""
        return None if times is None else _host(times, 6, "times")

    def cg(self, b, x, max_iter, tol, precond=True, times=None):
        """Returns (niters, normr, normr0); x is updated in place."""
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        check(lib().hpcgx_cg(self.h, self._v(b, 0, "b"), self._v(x, 0, "x"), int(max_iter),
                             float(tol), int(precond), C.byref(it), C.byref(nr), C.byref(nr0),
                             self._times(times)))
        return it.value, nr.value, nr0.value

    def cg_mixed(self, b, x, max_iter, tol, times=None):
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        check(lib().hpcgx_cg_mixed(self.h, self._v(b, 0, "b"), self._v(x, 0, "x"),
                                   int(max_iter), float(tol), C.byref(it), C.byref(nr),
                                   C.byref(nr0), self._times(times)))
        return it.value, nr.value, nr0.value

    def cg_host(self, b_host, x_host, max_iter, tol, mixed=False, precond=True, times=None):
        """Solve from host buffers (numpy or pinned CPU tensors); x_host updated."""
        self._pre()
        it, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        n = self.rows(0)
        mode = _lib.CG_MIXED if mixed else (_lib.CG_MG if precond else _lib.CG_PLAIN)
        check(lib().hpcgx_cg_host(self.h, mode, _host(b_host, n, "b_host"),
                                  _host(x_host, n, "x_host"), int(max_iter), float(tol),
                                  C.byref(it), C.byref(nr), C.byref(nr0), self._times(times)))
        return it.value, nr.value, nr0.value

    # ----------------------------------------------------------- adjoint
    def adjoint_grad(self, lam, x):
        self._pre()
        n = self.rows(0)
        g = torch.empty(n * STENCIL, dtype=torch.float64, device=self.device)
        check(lib().hpcgx_adjoint_grad(self.h, self._v(lam, 0, "lam"), self._v(x, 0, "x"),
                                       _ptr(g)))
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

    def _ptrs(self, ts, level, name):
        """One checked device pointer per rank (see _dev)."""
        if len(ts) != len(self.ranks):
            raise ValueError(f"{name}: {len(ts)} vectors for {len(self.ranks)} ranks")
        return (C.c_void_p * len(ts))(*[
            _dev(t, p.rows(level), F64, p.device, "%s[%d]" % (name, i)).value
            for i, (t, p) in enumerate(zip(ts, self.ranks))])

    def spmv(self, xs, level=0):
        self._pre()
        ys = [p.empty(level) for p in self.ranks]
        check(lib().hpcgx_group_spmv(self.g, level, self._ptrs(xs, level, "xs"),
                                     self._ptrs(ys, level, "ys")))
        return ys

    def symgs(self, rs, xs, level=0):
        """One symmetric sweep per slab (block Jacobi across slabs), x in place."""
        self._pre()
        check(lib().hpcgx_group_symgs(self.g, level, self._ptrs(rs, level, "rs"),
                                      self._ptrs(xs, level, "xs")))
        return xs

    def mg(self, rs):
        self._pre()
        xs = [p.empty(0) for p in self.ranks]
        check(lib().hpcgx_group_mg(self.g, self._ptrs(rs, 0, "rs"), self._ptrs(xs, 0, "xs")))
        return xs

    def cg(self, bs, xs, max_iter, tol, mode=_lib.CG_MG):
        """CG over the slabs; xs updated in place; returns (iters, normr, normr0)."""
        self._pre()
        k, nr, nr0 = C.c_int(), C.c_double(), C.c_double()
        check(lib().hpcgx_group_cg(self.g, mode, self._ptrs(bs, 0, "bs"), self._ptrs(xs, 0, "xs"),
                                   max_iter, tol,
                                   C.byref(k), C.byref(nr), C.byref(nr0)))
        return k.value, nr.value, nr0.value
