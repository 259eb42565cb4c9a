"""hpcg_b200 -- HPCG 3.1's multigrid-preconditioned CG iteration on B200 (sm_100a).

The compute path is libhpcgx.so (hand-written CUDA kernels behind the C ABI
of include/hpcgx.h).  ``Problem`` exposes the reference's operator set on
torch CUDA tensors; ``solve`` is the differentiable solve.
"""
from ._lib import HPCGXError, lib  # noqa: F401
from .problem import Group, Problem, check_status, nccl_unique_id  # noqa: F401
from .autograd import solve, symmetric_direction, varcoef_problem  # noqa: F401

__all__ = ["Problem", "Group", "nccl_unique_id", "check_status", "HPCGXError", "lib", "solve", "varcoef_problem", "symmetric_direction"]
