"""pastix_b200: a B200-native numerical phase for the PaStiX sparse direct solver.

The numerical factorization (POTRF / GETRF / SYTRF with static pivoting), the
supernodal triangular solves, the residual SpMV and the GMRES / CG / BiCGStab
refinement run as CUDA kernels for sm_100a behind PaStiX's own C API
(include/pastix_b200.h).  This package is the Python side: a ctypes mirror of
PaStiX's ``pypastix`` wrapper (:mod:`pastix_b200.pastix`), a minimal SpM
descriptor (:mod:`pastix_b200.spm`), the workload generators
(:mod:`pastix_b200.gen`) and the autograd adjoint (:mod:`pastix_b200.autograd`).
"""
from . import pastix, spm  # noqa: F401
from .pastix import PastixError, solver  # noqa: F401

__all__ = ["pastix", "spm", "solver", "PastixError"]
