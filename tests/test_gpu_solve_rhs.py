"""Solves with several right-hand sides (groups of 8 per CTA) against one
right-hand side at a time (the one-column kernels), for every factorization
kind in both precisions, and against the exact solution."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import analyse
from pastix_b200 import gen
from pastix_b200 import pastix as px

pytestmark = pytest.mark.gpu

# relative; the FP32 solves differ in summation order only
TOL = {False: 1e-12, True: 1e-5}
# forward error against x_true (FP32 factors: condition number x 6e-8)
FWD = {False: 1e-10, True: 1e-3}


@pytest.mark.parametrize("fact", ["POTRF", "SYTRF", "GETRF"])
@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("nrhs", [3, 16, 17])
def test_multi_rhs_matches_single(lib, fact, mixed, nrhs):
    if fact == "GETRF":
        A, grid = gen.convdiff27(14, 14, 14), (14, 14, 14)
    else:
        A, grid = gen.laplacian7(20, 20, 20), (20, 20, 20)
    pd, S, info = analyse(A, grid, fact, mixed=mixed)
    px.task_numfact(pd, S)
    n = A.shape[0]
    Af = S.full()
    xt = gen.rhs_uniform(n, nrhs, 5)
    B = torch.tensor(Af @ xt, device="cuda").t().contiguous().t()  # column major
    X = B.clone()
    px.solve_device(pd, X)
    torch.cuda.synchronize()
    for j in range(nrhs):
        xj = B[:, j].contiguous().clone()
        px.solve_device(pd, xj)
        torch.cuda.synchronize()
        err = (torch.linalg.norm(X[:, j] - xj) / torch.linalg.norm(xj)).item()
        assert err <= TOL[mixed], (j, err)
    Xh = X.cpu().numpy()
    assert np.linalg.norm(Xh - xt) / np.linalg.norm(xt) <= FWD[mixed]
    assert lib.pgpu_device_status(pd.ptr) == 0
