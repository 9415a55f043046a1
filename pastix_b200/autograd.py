"""Differentiable sparse solve: ``x = A(values)^{-1} b`` as a torch.autograd.Function.

Forward factorizes A with the given values on the GPU (pgpu_numfact_device)
and solves.  Backward reuses the resident factors: one transposed supernodal
solve ``lambda = A^{-T} g`` (U^T L^T for LU; the same factors for LL^T and
LDL^T), ``grad_b = lambda``, and the value gradient ``-lambda_i x_j`` over the
stored pattern from one sampled outer-product kernel (pgpu_sampled_outer); no
refactorization.  Only float64 CUDA tensors are accepted: the library has no
CPU path.

A solver holds one set of factors.  Each factorization bumps
``SparseSolver.version``; a forward records the version it solved with, and
its backward refactorizes from the values it saved when another forward has
replaced the factors in between, so the gradient always belongs to the
matrix of its own forward.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from . import pastix as px
from .spm import mtxtype, spmatrix


class SparseSolver:
    """Analysed pattern + GPU factors of a square sparse matrix.

    ``A`` gives the pattern (SciPy sparse); symmetric kinds store the lower
    triangle, so ``values`` follows ``self.spm.values`` order.  ``grid`` =
    (nx, ny, nz) uses the grid nested dissection (example/ordering_grid.c),
    otherwise the built-in ordering."""

    def __init__(self, A, factotype: str = "POTRF", grid=None, mixed: bool = False):
        self.factotype = factotype
        ip, dp = px.initParam()
        ip[px.iparm.factorization] = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}[factotype]
        ip[px.iparm.mixed] = 1 if mixed else 0
        self.pd = px.init(ip, dp)
        kind = mtxtype.General if factotype == "GETRF" else mtxtype.Symmetric
        self.spm = spmatrix(A, kind)
        if grid is not None:
            px.analyze_grid(self.pd, self.spm, *grid)
        else:
            px.task_analyze(self.pd, self.spm)
        self.n = self.spm.n
        self.nnz = self.spm.nnz
        self.version = 0  # bumped by every factorization


    def factorize(self, values: torch.Tensor) -> None:
        _check_cuda(values)
        if values.numel() != self.nnz:
            raise ValueError(f"values has {values.numel()} entries, the pattern {self.nnz}")
        torch.cuda.current_stream().synchronize()
        px.numfact_device(self.pd, values.contiguous())
        self.version += 1

    def solve(self, b: torch.Tensor, transposed: bool = False) -> torch.Tensor:
        """Device solve with the current factors (no autograd)."""
        _check_cuda(b)
        x = b.clone()
        if x.dim() == 2:
            x = x.t().contiguous().t()  # column major
        n = x.shape[0]
        nrhs = 1 if x.dim() == 1 else x.shape[1]
        ld = n if x.dim() == 1 else x.stride(1)
        fn = _lib.load().pgpu_solve_transposed_device if transposed else _lib.load().pgpu_solve_device
        rc = fn(self.pd.ptr, nrhs, C.c_void_p(x.data_ptr()), ld, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc:
            raise px.PastixError("pgpu_solve_device", rc)
        return x

    def sampled_outer(self, lam: torch.Tensor, x: torch.Tensor, alpha: float = -1.0) -> torch.Tensor:
        """G[e] = alpha * lam[row(e)] * x[col(e)] (+ the mirrored term for symmetric storage)."""
        G = torch.empty(self.nnz, dtype=torch.float64, device=lam.device)
        rc = _lib.load().pgpu_sampled_outer(self.pd.ptr, alpha, C.c_void_p(lam.data_ptr()), C.c_void_p(x.data_ptr()),
                                             C.c_void_p(G.data_ptr()),
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc:
            raise px.PastixError("pgpu_sampled_outer", rc)
        return G


def _check_cuda(t: torch.Tensor) -> None:
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError("pastix_b200 solves take float64 CUDA tensors (there is no CPU path)")


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, b, solver: SparseSolver):
        solver.factorize(values.detach())
        x = solver.solve(b.detach())
        ctx.solver = solver
        ctx.version = solver.version
        ctx.save_for_backward(x, values.detach())
        return x

    @staticmethod
    def backward(ctx, gx):
        x, values = ctx.saved_tensors
        solver: SparseSolver = ctx.solver
        if solver.version != ctx.version:
            # another forward factorized different values since: restore ours
            solver.factorize(values)
        gx = gx.contiguous()
        lam = solver.solve(gx, transposed=True)
        gvals = None
        if ctx.needs_input_grad[0]:
            if x.dim() == 1:
                gvals = solver.sampled_outer(lam, x)
            else:
                gvals = sum(solver.sampled_outer(lam[:, j].contiguous(), x[:, j].contiguous())
                            for j in range(x.shape[1]))
        return gvals, (lam if ctx.needs_input_grad[1] else None), None


def solve(values: torch.Tensor, b: torch.Tensor, solver: SparseSolver) -> torch.Tensor:
    """x = A(values)^{-1} b, differentiable in values and b."""
    return _Solve.apply(values, b, solver)
