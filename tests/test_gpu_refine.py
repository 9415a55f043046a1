"""GPU refinement: the reference's own integration cases (example/CTestLists.txt)
on its fixture matrices, mixed precision, and the refinement variants.

Known answers restated from the reference's tests:
  orsirr.rua  LU (-f 2) with GMRES and BiCGStab     (CTestLists.txt:121,148-149)
  small.rsa   LDL^T (-f 1), dparm_epsilon_magn_ctrl 1e-14, CG   (:117,147)
each solved to the refinement tolerance ||b - Ax|| / ||b|| <= 1e-12 (the
double-precision default of refinement/pastix_task_refine.c:133-141).
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sps

from conftest import ROOT, analyse, backward_error
from pastix_b200 import gen
from pastix_b200 import pastix as px
from pastix_b200.spm import mtxtype, spmatrix

pytestmark = pytest.mark.gpu


def _fixture(name):
    z = np.load(ROOT / "tests" / "golden" / f"{name}.npz")
    n = int(z["n"])
    A = sps.csc_matrix((z["values"], z["rowind"], z["colptr"]), shape=(n, n))
    return A, str(z["mxtype"])


def _solve_refine(A, kind, fact, refine, magn=0.0, mixed=False, nrhs=1, grid=None):
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}[fact]
    ip[px.iparm.refinement] = refine
    ip[px.iparm.mixed] = 1 if mixed else 0
    dp[px.dparm.epsilon_magn_ctrl] = magn
    dp[px.dparm.epsilon_refinement] = 1e-12
    pd = px.init(ip, dp)
    S = spmatrix(A, kind)
    if grid:
        px.analyze_grid(pd, S, *grid)
    else:
        px.task_analyze(pd, S)
    px.task_numfact(pd, S)
    Af = S.full()
    rng = np.random.default_rng(3)
    xt = np.asfortranarray(rng.uniform(-1, 1, (A.shape[0], nrhs)))
    b = np.asfortranarray(Af @ xt)
    x = b.copy(order="F")
    px.task_solve(pd, S, x)
    px.task_refine(pd, S, b, x)
    return Af, b, x, ip, dp


@pytest.mark.parametrize("refine", [px.refine.GMRES, px.refine.BiCGSTAB])
def test_orsirr_lu(lib, refine):
    A, mx = _fixture("orsirr")
    assert mx == "RUA"
    Af, b, x, ip, dp = _solve_refine(A, mtxtype.General, "GETRF", refine)
    for j in range(b.shape[1]):
        assert np.linalg.norm(b[:, j] - Af @ x[:, j]) / np.linalg.norm(b[:, j]) <= 1e-12


def test_small_rsa_ldlt_cg(lib):
    A, mx = _fixture("small")
    assert mx == "RSA"
    Af, b, x, ip, dp = _solve_refine(A, mtxtype.Symmetric, "SYTRF", px.refine.CG, magn=1e-14)
    r = np.linalg.norm(b[:, 0] - Af @ x[:, 0]) / np.linalg.norm(b[:, 0])
    assert r <= 1e-12, (r, ip[px.iparm.nbiter], ip[px.iparm.static_pivoting])


@pytest.mark.parametrize("refine", [px.refine.GMRES, px.refine.CG, px.refine.SR, px.refine.BiCGSTAB])
def test_mixed_precision_refinement(lib, refine):
    A = gen.laplacian7(24, 24, 24)
    Af, b, x, ip, dp = _solve_refine(A, mtxtype.Symmetric, "POTRF", refine, mixed=True, nrhs=2, grid=(24, 24, 24))
    for j in range(2):
        assert np.linalg.norm(b[:, j] - Af @ x[:, j]) / np.linalg.norm(b[:, j]) <= 1e-12
        assert backward_error(Af, x[:, j], b[:, j]) <= 1e-12
    assert 1 <= ip[px.iparm.nbiter] <= 30


def test_mixed_lu_gmres(lib):
    A, grid, _ = gen.workload("cd64", small=True)
    Af, b, x, ip, dp = _solve_refine(A, mtxtype.General, "GETRF", px.refine.GMRES, mixed=True, grid=grid)
    assert backward_error(Af, x[:, 0], b[:, 0]) <= 1e-12


def test_mixed_ldlt(lib):
    A, grid, _ = gen.workload("el48", small=True)
    Af, b, x, ip, dp = _solve_refine(A, mtxtype.Symmetric, "SYTRF", px.refine.GMRES, mixed=True, grid=grid)
    assert backward_error(Af, x[:, 0], b[:, 0]) <= 1e-12


def _refine_both(A, kind, fact, grid, nrhs, mixed, method=px.refine.GMRES):
    """pastix_task_refine on nrhs columns as one block (default) and with the
    column loop, from the same factors and the same first solve."""
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}[fact]
    ip[px.iparm.refinement] = method
    ip[px.iparm.mixed] = 1 if mixed else 0
    dp[px.dparm.epsilon_refinement] = 1e-12
    pd = px.init(ip, dp)
    S = spmatrix(A, kind)
    px.analyze_grid(pd, S, *grid)
    px.task_numfact(pd, S)
    Af = S.full()
    xt = np.asfortranarray(np.random.default_rng(8).uniform(-1, 1, (A.shape[0], nrhs)))
    b = np.asfortranarray(Af @ xt)
    x0 = b.copy(order="F")
    px.task_solve(pd, S, x0)
    out = {}
    for block in (True, False):
        px.refine_block(pd, block)
        x = x0.copy(order="F")
        px.task_refine(pd, S, b, x)
        out[block] = (x, int(ip[px.iparm.nbiter]))
    return Af, b, out


@pytest.mark.parametrize("name,kind,fact,nrhs,method", [
    ("cd64", mtxtype.General, "GETRF", 5, px.refine.GMRES),
    ("el48", mtxtype.Symmetric, "SYTRF", 9, px.refine.GMRES),
    ("lap100", mtxtype.Symmetric, "POTRF", 6, px.refine.CG),
    ("grf512", mtxtype.Symmetric, "POTRF", 3, px.refine.CG)])
def test_block_refinement_matches_columns(lib, name, kind, fact, nrhs, method):
    """The refinement block runs the per-column GMRES (z_refine_gmres.c) or CG
    (z_refine_grad.c) for every column at once: each column converges
    (backward error 1e-12) with the same iteration count as the column loop
    (one apart at most: the multi-column FP32 solve rounds differently) and to
    the same solution."""
    A, grid, _ = gen.workload(name, small=True)
    Af, b, out = _refine_both(A, kind, fact, grid, nrhs, mixed=True, method=method)
    (xb, itb), (xc, itc) = out[True], out[False]
    for j in range(nrhs):
        assert backward_error(Af, xb[:, j], b[:, j]) <= 1e-12
        assert backward_error(Af, xc[:, j], b[:, j]) <= 1e-12
    assert abs(itb - itc) <= 1
    # two solutions with backward error 1e-12 differ by up to cond(A) x 1e-12;
    # the shifted indefinite elasticity matrix has cond ~1e4-1e5
    assert np.linalg.norm(xb - xc) / np.linalg.norm(xc) <= (1e-9 if fact == "GETRF" else 1e-7)
