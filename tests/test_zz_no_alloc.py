"""pgpu_solve_device_static (the solve that allocates nothing) against
pgpu_solve_device, through the C ABI, on two calls in a row, with device
free memory unchanged across the calls that follow the first."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import analyse
from pastix_b200 import _lib, gen
from pastix_b200 import pastix as px

pytestmark = pytest.mark.gpu

# relative; both solves scatter with atomics, so the last bits may differ:
# FP64 factors agree to 1e-12, FP32 factors (mixed precision) to FP32 rounding
TOL = {False: 1e-12, True: 1e-5}


def _solve(fn, pd, B):
    X = B.clone().t().contiguous().t()  # column major
    n = X.shape[0]
    rc = fn(pd.ptr, X.shape[1], C.c_void_p(X.data_ptr()), n, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    return X


@pytest.mark.parametrize("fact,mixed", [("POTRF", False), ("GETRF", False), ("SYTRF", True)])
def test_static_solve_matches(lib, fact, mixed):
    if fact == "GETRF":
        A, grid = gen.convdiff27(12, 12, 12), (12, 12, 12)
    else:
        A, grid = gen.laplacian7(16, 16, 16), (16, 16, 16)
    pd, S, info = analyse(A, grid, fact, mixed=mixed)
    px.task_numfact(pd, S)
    l = _lib.load()
    n = A.shape[0]
    g = torch.Generator(device="cuda").manual_seed(7)
    B = torch.rand(n, 3, dtype=torch.float64, device="cuda", generator=g) - 0.5
    # the static solve runs first on this freshly factorized instance, so the
    # work areas of pgpu_solve_device do not exist yet; after the first call
    # (the per-device set-up) device memory must not change
    X0 = _solve(l.pgpu_solve_device_static, pd, B)
    Xs = [B.clone().t().contiguous().t() for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for X in Xs:
        rc = l.pgpu_solve_device_static(pd.ptr, X.shape[1], C.c_void_p(X.data_ptr()), n,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ref = _solve(l.pgpu_solve_device, pd, B)
    for X in [X0] + Xs:
        err = torch.linalg.norm(X - ref) / torch.linalg.norm(ref)
        assert err.item() <= TOL[mixed], err.item()
    assert l.pgpu_device_status(pd.ptr) == 0


def test_static_solve_rejects_large(lib):
    A, grid = gen.laplacian7(10, 10, 10), (10, 10, 10)
    pd, S, info = analyse(A, grid, "POTRF")
    px.task_numfact(pd, S)
    l = _lib.load()
    n = A.shape[0]
    nrhs = 1048576 // n + 1  # one column more than the fixed array holds
    B = torch.zeros(n, nrhs, dtype=torch.float64, device="cuda").t().contiguous().t()
    rc = l.pgpu_solve_device_static(pd.ptr, nrhs, C.c_void_p(B.data_ptr()), n, None)
    assert rc == px.error.BADPARAMETER
    assert torch.count_nonzero(B).item() == 0
