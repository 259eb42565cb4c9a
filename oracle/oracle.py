"""ctypes bindings for the checker libraries built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY.  ``Oracle`` wraps the C restatement of HPCG 3.1's
reference path (``_build/liboracle.so``); ``RefProblem`` wraps the reference's
own ``_ref`` code compiled from its sources (``_ref/libhpcgref.so``).  Only
tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product in hpcg_b200/ never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIBREF = os.path.join(HERE, "_ref", "libhpcgref.so")
XHPCG_REF = os.path.join(HERE, "_ref", "xhpcg")
STENCIL = 27
LEVELS = 4

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double


def build(quiet: bool = True) -> None:
    """Runs oracle/Makefile (the reference part only where its sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a):
    if a is None:
        return None
    if not a.flags.c_contiguous:
        raise ValueError("oracle arrays must be C-contiguous")
    return a.ctypes.data_as(_P)


class _Level(C.Structure):
    _fields_ = [("nrow", _I64), ("nnz", _P), ("cols", _P), ("vals", _P), ("diag", _P),
                ("order", _P), ("f2c", _P), ("nc", _I64), ("Axf", _P), ("rc", _P),
                ("xc", _P), ("slab_rows", _I64)]


class Level:
    """One level in the contiguous 27-slot layout (numpy arrays)."""

    def __init__(self, nx, ny, nz, nnz, cols, vals, diag, f2c=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nrow = nx * ny * nz
        self.nnz, self.cols, self.vals, self.diag, self.f2c = nnz, cols, vals, diag, f2c
        self.order = None        # SYMGS visiting order (int64) or None
        self.position = None     # natural row -> position in colour order
        self.slab_rows = 0       # z-slab decomposition: rows per rank (0: one rank)

    @property
    def vals_bf16(self):
        if not hasattr(self, "_bf16"):
            self._bf16 = np.empty(self.vals.shape, np.uint16)
            Oracle.lib().or_vals_to_bf16(self.vals.size, _ptr(self.vals), _ptr(self._bf16))
        return self._bf16


def geometric_colour(nx, ny, nz):
    """colour = (ix&1) + 2(iy&1) + 4(iz&1): the colouring the reference's
    greedy algorithm produces on the 27-point stencil."""
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return ((ix & 1) + 2 * (iy & 1) + 4 * (iz & 1)).reshape(-1).astype(np.int32)


class Oracle:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(LIBORACLE):
                build()
            lib = C.CDLL(LIBORACLE)
            lib.or_generate_problem.restype = _I64
            lib.or_generate_varcoef.restype = _I64
            lib.or_dot.restype = _D
            lib.or_residual.restype = _D
            lib.or_uniform.restype = _D
            lib.or_normal.restype = _D
            lib.or_splitmix64.restype = C.c_uint64
            lib.or_splitmix64.argtypes = [C.c_uint64]
            lib.or_uniform.argtypes = [C.c_uint64, C.c_uint64]
            lib.or_normal.argtypes = [C.c_uint64, C.c_uint64]
            lib.or_fill_uniform.argtypes = [C.c_uint64, _I64, _D, _D, _P]
            lib.or_fill_normal.argtypes = [C.c_uint64, _I64, _P]
            lib.or_generate_varcoef.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                                _D, _P, _P, _P, _P]
            lib.or_waxpby.argtypes = [_I64, _D, _P, _D, _P, _P]
            lib.or_dot.argtypes = [_I64, _P, _P]
            lib.or_dot_slab.restype = _D
            lib.or_dot_slab.argtypes = [_I64, _P, _P, _I64]
            lib.or_residual.argtypes = [_I64, _P, _P]
            lib.or_bf16_from_double.restype = C.c_uint16
            lib.or_bf16_from_double.argtypes = [_D]
            lib.or_vals_to_bf16.argtypes = [_I64, _P, _P]
            lib.or_cg.argtypes = [_P, C.c_int, _P, _P, C.c_int, _D, C.c_int,
                                  C.POINTER(C.c_int), C.POINTER(_D), C.POINTER(_D), _P]
            lib.or_fcg.argtypes = [_P, _P, C.c_int, _P, _P, C.c_int, _D,
                                   C.POINTER(C.c_int), C.POINTER(_D), C.POINTER(_D), _P, _P]
            lib.or_mg.argtypes = [_P, C.c_int, _P, _P]
            lib.or_mg32.argtypes = [_P, C.c_int, _P, _P, _P]
            lib.or_greedy_colour.argtypes = [_I64, _P, _P, _P, _P]
            for f in ("or_stencil_spmv", "or_stencil_symgs", "or_stencil_symgs32"):
                getattr(lib, f).argtypes = [C.c_int, C.c_int, C.c_int, _P, _P]
            cls._lib = lib
        return cls._lib

    # ------------------------------------------------------------ problems
    @classmethod
    def generate(cls, nx, ny, nz):
        n = nx * ny * nz
        nnz = np.zeros(n, np.uint8)
        cols = np.zeros(n * STENCIL, np.int32)
        vals = np.zeros(n * STENCIL, np.float64)
        diag = np.zeros(n, np.int32)
        b, x, xe = np.zeros(n), np.zeros(n), np.zeros(n)
        cls.lib().or_generate_problem(nx, ny, nz, _ptr(nnz), _ptr(cols), _ptr(vals), _ptr(diag),
                                      _ptr(b), _ptr(x), _ptr(xe))
        return Level(nx, ny, nz, nnz, cols, vals, diag), b, x, xe

    @classmethod
    def generate_varcoef(cls, nx, ny, nz, seed, sigma, level=0):
        n = nx * ny * nz
        nnz = np.zeros(n, np.uint8)
        cols = np.zeros(n * STENCIL, np.int32)
        vals = np.zeros(n * STENCIL, np.float64)
        diag = np.zeros(n, np.int32)
        cls.lib().or_generate_varcoef(nx, ny, nz, level, seed, sigma, _ptr(nnz), _ptr(cols),
                                      _ptr(vals), _ptr(diag))
        return Level(nx, ny, nz, nnz, cols, vals, diag)

    @classmethod
    def f2c(cls, nx, ny, nz):
        f = np.zeros((nx // 2) * (ny // 2) * (nz // 2), np.int32)
        cls.lib().or_f2c(nx, ny, nz, _ptr(f))
        return f

    @classmethod
    def hierarchy(cls, nx, ny, nz, levels=LEVELS, varcoef=None):
        """The reference's 4-level hierarchy (src/main.cpp:139-145).  With
        varcoef=(seed, sigma) the levels hold the variable-coefficient matrix
        and its coarse versions (or_generate_varcoef's level rule)."""
        L = []
        b = x = xe = None
        for l in range(levels):
            if varcoef is None:
                lev, bb, xx, xxe = cls.generate(nx, ny, nz)
                if l == 0:
                    b, x, xe = bb, xx, xxe
            else:
                lev = cls.generate_varcoef(nx, ny, nz, varcoef[0], varcoef[1], level=l)
            if l + 1 < levels:
                lev.f2c = cls.f2c(nx, ny, nz)
            L.append(lev)
            nx, ny, nz = nx // 2, ny // 2, nz // 2
        return L, b, x, xe

    @classmethod
    def slab_hierarchy(cls, nx, ny, nz, nranks, levels=LEVELS):
        """The hierarchy of a z-slab decomposition into nranks slabs of nz planes
        (a 1 x 1 x nranks process grid, src/GenerateGeometry.cpp:49-169): the
        global grid nx x ny x (nz nranks) and its injection, every slab
        coarsening its own planes (src/GenerateCoarseProblem.cpp:52), with
        .slab_rows set on every level for the block-Jacobi smoother and the
        per-rank dot products."""
        L, b, x, xe = cls.hierarchy(nx, ny, nz * nranks, levels)
        for l, lev in enumerate(L):
            lev.slab_rows = (nx >> l) * (ny >> l) * (nz >> l) if nranks > 1 else 0
        return L, b, x, xe

    @classmethod
    def colour_order(cls, L):
        """Greedy colouring (src/OptimizeProblem.cpp:43-96) on every level;
        sets .position (natural -> colour order) and .order (its inverse)."""
        for lev in L:
            colors = np.zeros(lev.nrow, np.int32)
            pos = np.zeros(lev.nrow, np.int64)
            ncol = cls.lib().or_greedy_colour(lev.nrow, _ptr(lev.nnz), _ptr(lev.cols),
                                              _ptr(colors), _ptr(pos))
            lev.colors, lev.ncolors = colors, ncol
            lev.position = pos
            order = np.empty(lev.nrow, np.int64)
            order[pos] = np.arange(lev.nrow, dtype=np.int64)
            lev.order = order
        return L

    # ------------------------------------------------------------ kernels
    @classmethod
    def spmv(cls, lev, x):
        y = np.zeros(lev.nrow)
        cls.lib().or_spmv(_I64(lev.nrow), _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals), _ptr(x),
                          _ptr(y))
        return y

    @classmethod
    def spmv32(cls, lev, x32):
        y = np.zeros(lev.nrow, np.float32)
        cls.lib().or_spmv32(_I64(lev.nrow), _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals_bf16),
                            _ptr(x32), _ptr(y))
        return y

    @classmethod
    def symgs(cls, lev, r, x, coloured=False):
        x = x.copy()
        order = lev.order if coloured else None
        cls.lib().or_symgs_slab(_I64(lev.nrow), _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals),
                                _ptr(lev.diag), _ptr(order), _I64(lev.slab_rows), _ptr(r),
                                _ptr(x))
        return x

    @classmethod
    def symgs32(cls, lev, r, x32, coloured=True):
        x32 = x32.astype(np.float32).copy()
        order = lev.order if coloured else None
        r64 = r if r.dtype == np.float64 else None
        r32 = r if r.dtype == np.float32 else None
        cls.lib().or_symgs32(_I64(lev.nrow), _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals_bf16),
                             _ptr(lev.diag), _ptr(order), _ptr(r64), _ptr(r32), _ptr(x32))
        return x32

    @classmethod
    def restriction(cls, f2c, rf, Axf):
        rc = np.zeros(f2c.size)
        cls.lib().or_restriction(_I64(f2c.size), _ptr(f2c), _ptr(rf), _ptr(Axf), _ptr(rc))
        return rc

    @classmethod
    def prolongation(cls, f2c, xc, xf):
        xf = xf.copy()
        cls.lib().or_prolongation(_I64(f2c.size), _ptr(f2c), _ptr(xc), _ptr(xf))
        return xf

    @classmethod
    def dot(cls, x, y, slab_rows=0):
        return cls.lib().or_dot_slab(x.size, _ptr(x), _ptr(y), slab_rows)

    @classmethod
    def waxpby(cls, alpha, x, beta, y):
        w = np.zeros_like(x)
        cls.lib().or_waxpby(x.size, alpha, _ptr(x), beta, _ptr(y), _ptr(w))
        return w

    @classmethod
    def residual(cls, v1, v2):
        return cls.lib().or_residual(v1.size, _ptr(v1), _ptr(v2))

    @staticmethod
    def _levels(L, coloured):
        arr = (_Level * len(L))()
        keep = []
        for i, lev in enumerate(L):
            nc = lev.f2c.size if lev.f2c is not None else 0
            Axf, rc, xc = np.zeros(lev.nrow), np.zeros(max(nc, 1)), np.zeros(max(nc, 1))
            keep += [Axf, rc, xc]
            arr[i] = _Level(lev.nrow, _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals), _ptr(lev.diag),
                            _ptr(lev.order) if coloured else None, _ptr(lev.f2c), nc, _ptr(Axf),
                            _ptr(rc), _ptr(xc), lev.slab_rows)
        return arr, keep

    @staticmethod
    def _levels32(L, coloured):
        arr = (_Level * len(L))()
        keep = []
        for i, lev in enumerate(L):
            nc = lev.f2c.size if lev.f2c is not None else 0
            Axf = np.zeros(lev.nrow, np.float32)
            rc, xc = np.zeros(max(nc, 1), np.float32), np.zeros(max(nc, 1), np.float32)
            keep += [Axf, rc, xc]
            arr[i] = _Level(lev.nrow, _ptr(lev.nnz), _ptr(lev.cols), _ptr(lev.vals_bf16),
                            _ptr(lev.diag), _ptr(lev.order) if coloured else None, _ptr(lev.f2c),
                            nc, _ptr(Axf), _ptr(rc), _ptr(xc), lev.slab_rows)
        return arr, keep

    @classmethod
    def mg(cls, L, r, coloured=False):
        arr, keep = cls._levels(L, coloured)
        x = np.zeros(L[0].nrow)
        err = cls.lib().or_mg(arr, len(L), _ptr(r), _ptr(x))
        assert err == 0
        return x

    @classmethod
    def mg32(cls, L, r64, coloured=True):
        arr, keep = cls._levels32(L, coloured)
        x = np.zeros(L[0].nrow, np.float32)
        err = cls.lib().or_mg32(arr, len(L), _ptr(r64), None, _ptr(x))
        assert err == 0
        return x

    @classmethod
    def cg(cls, L, b, x0, max_iter, tol, precond=True, coloured=False):
        arr, keep = cls._levels(L, coloured)
        x = x0.copy()
        work = np.zeros(4 * L[0].nrow)
        it, nr, nr0 = C.c_int(0), _D(0), _D(0)
        err = cls.lib().or_cg(arr, len(L), _ptr(b), _ptr(x), max_iter, tol, int(precond),
                              C.byref(it), C.byref(nr), C.byref(nr0), _ptr(work))
        assert err == 0
        return x, it.value, nr.value, nr0.value

    @classmethod
    def fcg(cls, L, b, x0, max_iter, tol):
        arr, keep = cls._levels(L, True)
        arr32, keep32 = cls._levels32(L, True)
        x = x0.copy()
        work = np.zeros(4 * L[0].nrow)
        z32 = np.zeros(L[0].nrow, np.float32)
        it, nr, nr0 = C.c_int(0), _D(0), _D(0)
        err = cls.lib().or_fcg(arr, arr32, len(L), _ptr(b), _ptr(x), max_iter, tol, C.byref(it),
                               C.byref(nr), C.byref(nr0), _ptr(work), _ptr(z32))
        assert err == 0
        return x, it.value, nr.value, nr0.value

    # ------------------------------------------------- matrix-free (large grids)
    @classmethod
    def stencil_spmv(cls, dims, x):
        """ComputeSPMV_ref on the reference problem of an nx x ny x nz grid,
        rows generated on the fly (bit-identical to ``spmv``)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        cls.lib().or_stencil_spmv(*dims, _ptr(x), _ptr(y))
        return y

    @classmethod
    def stencil_symgs(cls, dims, r, x):
        """ComputeSYMGS_ref in colour order on the reference problem
        (bit-identical to ``symgs(..., coloured=True)``)."""
        x = np.array(x, dtype=np.float64)
        cls.lib().or_stencil_symgs(*dims, _ptr(np.ascontiguousarray(r, dtype=np.float64)), _ptr(x))
        return x

    @classmethod
    def stencil_symgs32(cls, dims, r64, x32):
        """The mixed FP32/BF16 sweep in colour order on the reference problem
        (bit-identical to ``symgs32`` with an FP64 right-hand side)."""
        x = np.array(x32, dtype=np.float32)
        cls.lib().or_stencil_symgs32(*dims, _ptr(np.ascontiguousarray(r64, dtype=np.float64)),
                                     _ptr(x))
        return x

    @classmethod
    def adjoint_grad(cls, lev, lam, x):
        g = np.zeros(lev.nrow * STENCIL)
        cls.lib().or_adjoint_grad(_I64(lev.nrow), _ptr(lev.nnz), _ptr(lev.cols), _ptr(lam),
                                  _ptr(x), _ptr(g))
        return g

    # ------------------------------------------------------------ inputs
    @classmethod
    def uniform(cls, seed, n, lo=0.0, hi=1.0):
        v = np.zeros(n)
        cls.lib().or_fill_uniform(seed, n, lo, hi, _ptr(v))
        return v

    @classmethod
    def normal(cls, seed, n):
        v = np.zeros(n)
        cls.lib().or_fill_normal(seed, n, _ptr(v))
        return v


class RefProblem:
    """The reference's own problem and _ref kernels (oracle/_ref/libhpcgref.so)."""
    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(LIBREF)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(LIBREF)
            lib.ref_create.restype = _P
            lib.ref_create.argtypes = [C.c_int, C.c_int, C.c_int]
            lib.ref_create_levels.restype = _P
            lib.ref_create_levels.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
            lib.ref_destroy.argtypes = [_P]
            lib.ref_level_rows.restype = _I64
            lib.ref_level_rows.argtypes = [_P, C.c_int]
            lib.ref_level_nnz.restype = _I64
            lib.ref_level_nnz.argtypes = [_P, C.c_int]
            lib.ref_export_level.argtypes = [_P, C.c_int, _P, _P, _P, _P, _P]
            lib.ref_get_vectors.argtypes = [_P, _P, _P, _P]
            lib.ref_replace_diagonal.argtypes = [_P, C.c_int, _P]
            lib.ref_set_level_values.argtypes = [_P, C.c_int, _P]
            for f in ("ref_spmv", "ref_symgs", "ref_symgs_permuted"):
                getattr(lib, f).argtypes = [_P, C.c_int, _P, _P]
            lib.ref_mg.argtypes = [_P, _P, _P]
            lib.ref_mg_permuted.argtypes = [_P, _P, _P]
            lib.ref_restriction.argtypes = [_P, C.c_int, _P, _P, _P]
            lib.ref_prolongation.argtypes = [_P, C.c_int, _P, _P]
            lib.ref_dot.restype = _D
            lib.ref_dot.argtypes = [_I64, _P, _P]
            lib.ref_waxpby.argtypes = [_I64, _D, _P, _D, _P, _P]
            lib.ref_residual.restype = _D
            lib.ref_residual.argtypes = [_I64, _P, _P]
            lib.ref_cg.argtypes = [_P, _P, _P, C.c_int, _D, C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(_D), C.POINTER(_D), _P]
            lib.ref_build_permuted.argtypes = [_P, _P]
            lib.ref_cg_permuted.argtypes = [_P, _P, _P, C.c_int, _D, C.c_int, C.POINTER(C.c_int),
                                            C.POINTER(_D), C.POINTER(_D)]
            lib.ref_wtime.restype = _D
            cls._lib = lib
        return cls._lib

    def __init__(self, nx, ny, nz, levels=LEVELS):
        """The reference's set-up (src/main.cpp:116-159) with ``levels``
        levels; every level but the last needs even dimensions."""
        self.h = None
        self.levels = levels
        self.h = self.lib().ref_create_levels(nx, ny, nz, levels)
        if not self.h:
            raise ValueError("levels must be 1..%d" % LEVELS)
        self.dims = [(nx >> l, ny >> l, nz >> l) for l in range(levels)]

    def close(self):
        if self.h:
            self.lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rows(self, level=0):
        return self.lib().ref_level_rows(self.h, level)

    def export_level(self, level):
        n = self.rows(level)
        nnz = np.zeros(n, np.uint8)
        cols = np.zeros(n * STENCIL, np.int32)
        vals = np.zeros(n * STENCIL)
        diag = np.zeros(n, np.int32)
        f2c = np.zeros(self.rows(level + 1), np.int32) if level + 1 < self.levels else None
        self.lib().ref_export_level(self.h, level, _ptr(nnz), _ptr(cols), _ptr(vals), _ptr(diag),
                                    _ptr(f2c))
        nx, ny, nz = self.dims[level]
        return Level(nx, ny, nz, nnz, cols, vals, diag, f2c)

    def vectors(self):
        n = self.rows(0)
        b, x, xe = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib().ref_get_vectors(self.h, _ptr(b), _ptr(x), _ptr(xe))
        return b, x, xe

    def replace_diagonal(self, level, d):
        self.lib().ref_replace_diagonal(self.h, level, _ptr(np.ascontiguousarray(d)))

    def set_level_values(self, level, vals):
        self.lib().ref_set_level_values(self.h, level, _ptr(np.ascontiguousarray(vals)))

    def spmv(self, level, x):
        y = np.zeros(self.rows(level))
        assert self.lib().ref_spmv(self.h, level, _ptr(x), _ptr(y)) == 0
        return y

    def symgs(self, level, r, x):
        x = x.copy()
        assert self.lib().ref_symgs(self.h, level, _ptr(r), _ptr(x)) == 0
        return x

    def build_permuted(self, positions):
        pos = [np.ascontiguousarray(p, np.int64) for p in positions]
        arr = (_P * len(pos))(*[p.ctypes.data for p in pos])
        self._pos_keep = pos
        assert self.lib().ref_build_permuted(self.h, arr) == 0

    def symgs_permuted(self, level, r, x):
        x = x.copy()
        assert self.lib().ref_symgs_permuted(self.h, level, _ptr(r), _ptr(x)) == 0
        return x

    def mg(self, r):
        x = np.zeros(self.rows(0))
        assert self.lib().ref_mg(self.h, _ptr(r), _ptr(x)) == 0
        return x

    def mg_permuted(self, r):
        x = np.zeros(self.rows(0))
        assert self.lib().ref_mg_permuted(self.h, _ptr(r), _ptr(x)) == 0
        return x

    def restriction(self, level, rf, Axf):
        rc = np.zeros(self.rows(level + 1))
        assert self.lib().ref_restriction(self.h, level, _ptr(rf), _ptr(Axf), _ptr(rc)) == 0
        return rc

    def prolongation(self, level, xc, xf):
        xf = xf.copy()
        assert self.lib().ref_prolongation(self.h, level, _ptr(xc), _ptr(xf)) == 0
        return xf

    def dot(self, x, y):
        return self.lib().ref_dot(x.size, _ptr(x), _ptr(y))

    def waxpby(self, alpha, x, beta, y):
        w = np.zeros_like(x)
        assert self.lib().ref_waxpby(x.size, alpha, _ptr(x), beta, _ptr(y), _ptr(w)) == 0
        return w

    def residual(self, v1, v2):
        return self.lib().ref_residual(v1.size, _ptr(v1), _ptr(v2))

    def cg(self, b, x0, max_iter, tol, precond=True):
        x = x0.copy()
        it, nr, nr0 = C.c_int(0), _D(0), _D(0)
        times = np.zeros(10)
        assert self.lib().ref_cg(self.h, _ptr(b), _ptr(x), max_iter, tol, int(precond),
                                 C.byref(it), C.byref(nr), C.byref(nr0), _ptr(times)) == 0
        return x, it.value, nr.value, nr0.value, times

    def cg_permuted(self, b, x0, max_iter, tol, precond=True):
        x = x0.copy()
        it, nr, nr0 = C.c_int(0), _D(0), _D(0)
        assert self.lib().ref_cg_permuted(self.h, _ptr(b), _ptr(x), max_iter, tol, int(precond),
                                          C.byref(it), C.byref(nr), C.byref(nr0)) == 0
        return x, it.value, nr.value, nr0.value

    def wtime(self):
        return self.lib().ref_wtime()
