"""ctypes binding of libhpcgx.so (declarations in include/hpcgx.h).

The library is loaded from this package directory only.  There is no
fallback: if libhpcgx.so is missing or fails to load, importing the product
raises, so a CPU path can never stand in for the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# HPCGX_LIBRARY=checked selects the index-checked build (libhpcgx_checked.so)
LIB_PATH = os.path.join(HERE, "libhpcgx_checked.so" if os.environ.get("HPCGX_LIBRARY") == "checked"
                        else "libhpcgx.so")

_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_U64 = C.c_uint64
_D = C.c_double
_IP = C.POINTER(C.c_int)
_DP = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)

# hpcgx_halo_fn / hpcgx_sum_fn (include/hpcgx.h)
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_int64, C.c_int, C.c_void_p)
SUM_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)

# name -> (restype, argtypes); mirrors include/hpcgx.h
SIGNATURES = {
    "hpcgx_last_error": (C.c_char_p, []),
    "hpcgx_version": (_I, []),
    "hpcgx_init_device": (_I, [_I]),
    "hpcgx_create": (_I, [_I, _I, _I, _I, _I, C.POINTER(_P)]),
    "hpcgx_destroy": (_I, [_P]),
    "hpcgx_load_level": (_I, [_P, _I, _P, _P, _P]),
    "hpcgx_load_level_rows": (_I, [_P, _I, _P, _P, _P]),
    "hpcgx_check_f2c": (_I, [_P, _I, _P, _I64]),
    "hpcgx_generate": (_I, [_P, _I, _U64, _D]),
    "hpcgx_create_general": (_I, [_I, _I, _P]),
    "hpcgx_load_level_general": (_I, [_P, _I, _I64, _P, _P, _P, _P, _I64]),
    "hpcgx_colours": (_I, [_P, _I]),
    "hpcgx_build_mixed": (_I, [_P]),
    "hpcgx_set_stencil_columns": (_I, [_P, _I]),
    "hpcgx_set_diagonal_host": (_I, [_P, _I, _P]),
    "hpcgx_get_diagonal_host": (_I, [_P, _I, _P]),
    "hpcgx_set_values": (_I, [_P, _I, _P, _I]),
    "hpcgx_get_values": (_I, [_P, _I, _P, _P]),
    "hpcgx_memory_bytes": (_I, [_P, _DP]),
    "hpcgx_rows": (_I64, [_P, _I]),
    "hpcgx_spmv": (_I, [_P, _I, _P, _P]),
    "hpcgx_spmv_stencil": (_I, [_P, _I, _P, _P]),
    "hpcgx_symgs": (_I, [_P, _I, _P, _P]),
    "hpcgx_mg": (_I, [_P, _P, _P]),
    "hpcgx_restriction": (_I, [_P, _I, _P, _P, _P]),
    "hpcgx_prolongation": (_I, [_P, _I, _P, _P]),
    "hpcgx_dot": (_I, [_P, _I64, _P, _P, _DP]),
    "hpcgx_waxpby": (_I, [_P, _I64, _D, _P, _D, _P, _P]),
    "hpcgx_residual": (_I, [_P, _I64, _P, _P, _DP]),
    "hpcgx_dot_noalloc": (_I, [_I64, _P, _P, _P, _P]),
    "hpcgx_spmv_host": (_I, [_P, _I, _P, _P]),
    "hpcgx_symgs_host": (_I, [_P, _I, _P, _P]),
    "hpcgx_mg_host": (_I, [_P, _P, _P]),
    "hpcgx_dot_host": (_I, [_P, _I64, _P, _P, _DP]),
    "hpcgx_waxpby_host": (_I, [_P, _I64, _D, _P, _D, _P, _P]),
    "hpcgx_spmv_mixed": (_I, [_P, _I, _P, _P]),
    "hpcgx_symgs_mixed": (_I, [_P, _I, _P, _P, _P]),
    "hpcgx_mg_mixed": (_I, [_P, _P, _P]),
    "hpcgx_cg": (_I, [_P, _P, _P, _I, _D, _I, _IP, _DP, _DP, _P]),
    "hpcgx_cg_mixed": (_I, [_P, _P, _P, _I, _D, _IP, _DP, _DP, _P]),
    "hpcgx_cg_host": (_I, [_P, _I, _P, _P, _I, _D, _IP, _DP, _DP, _P]),
    "hpcgx_adjoint_grad": (_I, [_P, _P, _P, _P]),
    "hpcgx_fill_uniform": (_I, [_P, _I64, _U64, _D, _D, _P]),
    "hpcgx_fill_normal": (_I, [_P, _I64, _U64, _U64, _P]),
    "hpcgx_set_probe": (_I, [_P, _I]),
    "hpcgx_probe_read": (_I, [_P, _I, _DP, _I64P, _DP, _I]),
    "hpcgx_launch_count": (_I64, [_P]),
    "hpcgx_iteration_bytes": (_I, [_P, _I, _DP]),
    "hpcgx_synchronize": (_I, [_P]),
    "hpcgx_set_stream": (_I, [_P, _P]),
    "hpcgx_create_slab": (_I, [_I, _I, _I, _I, _I, _I, _I, C.POINTER(_P)]),
    "hpcgx_nccl_unique_id": (_I, [_P, _I]),
    "hpcgx_attach_nccl": (_I, [_P, _P, _I]),
    "hpcgx_attach_comm": (_I, [_P, HALO_FN, SUM_FN, _P]),
    "hpcgx_check_status": (_I, []),
    "hpcgx_group_create": (_I, [_P, _I, C.POINTER(_P)]),
    "hpcgx_group_destroy": (_I, [_P]),
    "hpcgx_group_spmv": (_I, [_P, _I, _P, _P]),
    "hpcgx_group_symgs": (_I, [_P, _I, _P, _P]),
    "hpcgx_group_mg": (_I, [_P, _P, _P]),
    "hpcgx_group_cg": (_I, [_P, _I, _P, _P, _I, _D, _IP, _DP, _DP]),
}

HPCGX_OK = 0
ERRORS = {1: "EINVAL", 2: "ECUDA", 3: "ESTATE", 4: "ENONFINITE", 5: "ELAYOUT", 6: "ENOMEM",
          7: "ECOMM", 8: "ETIMEOUT", 9: "ECHECK"}
NCCL_ID_BYTES = 128
GEN_HPCG, GEN_VARCOEF = 0, 1
PROBE_NONE, PROBE_GS_FINE, PROBE_SPMV_FINE, PROBE_GS_FINE_BWD = 0, 1, 2, 4
CG_PLAIN, CG_MG, CG_MIXED = 0, 1, 2


class HPCGXError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"hpcgx error {code} ({ERRORS.get(code, '?')}): {message}")
        self.code = code


_lib = None


def lib():
    """Loads libhpcgx.so once; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m hpcg_b200.build` "
                              "(nvcc, sm_100a) before using the CUDA path")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(rc: int) -> None:
    if rc != HPCGX_OK:
        raise HPCGXError(rc, lib().hpcgx_last_error().decode(errors="replace"))
