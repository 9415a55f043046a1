"""GPU parity with the reference PaStiX itself (oracle/_ref, compiled from its
sources), through the C ABI.

* The GPU consumes the reference's own analysis: the reference orders (the
  fixtures get a nested-dissection permutation and the reference finds its
  supernodes), and the SolverMatrix it produces is imported with
  pgpu_set_symbol.  Static-pivot counts must be equal -- 4997 for the
  reference's LDL^T test of small.rsa with magnitude control 1e-14
  (example/CTestLists.txt:117), 191 for an LU of orsirr.rua with a threshold
  of 1e-3 ||A||_F that makes the sign-keeping replacement of
  kernels/core_zgetrfsp.c:81-89 fire -- and the FP64 factors agree to 1e-12
  relative Frobenius.
* On the grid configurations the product's own analysis is the reference's
  (checked here again on the full-size grids), and the GPU factors are
  compared with the reference's static-scheduler factors at full size: the
  100^3 Laplacian (n = 10^6) and the 512^2 diffusion, the 27-point
  convection-diffusion LU at 32^3 and the elastic LDL^T at 24^3 nodes.
* FP32 factors (IPARM_MIXED) against the reference's own FP32 factorization,
  to FP32 accuracy.
The shifted indefinite elastic matrix factored by LDL^T without pivoting
(element growth ~1.4e3) amplifies rounding: at 24^3 nodes two CPU codes --
the reference and the oracle's restatement -- already differ by 2.4e-12, so
its bar is 1e-11.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import analyse, fixture_matrix
from pastix_b200 import gen
from pastix_b200 import pastix as px
from pastix_b200.spm import mtxtype, spmatrix

pytestmark = pytest.mark.gpu

FACT_ID = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}
NTHREADS = max(1, min(32, os.cpu_count() or 1))


def _expanded(perm, n):
    perm = np.asarray(perm)
    dof = n // perm.size
    return perm if dof == 1 else (perm[:, None] * dof + np.arange(dof)).ravel()


def _product_perm(A, fact):
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = FACT_ID[fact]
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    px.task_analyze(pd, S)
    return np.asarray(px.solver_info(pd)["permtab"]).copy()


def _gpu_on_reference_structure(r, A, fact, magn=0.0, mixed=False):
    s = r.structure()
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = FACT_ID[fact]
    ip[px.iparm.mixed] = 1 if mixed else 0
    dp[px.dparm.epsilon_magn_ctrl] = magn
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    px.set_symbol(pd, S, _expanded(s["permtab"], A.shape[0]), s["cb_fcol"], s["cb_lcol"], s["cb_fblok"],
                  s["bk_frow"], s["bk_lrow"], s["bk_fcblk"])
    px.task_numfact(pd, S)
    return pd, S


def _check_factors(r, pd, fact, tol):
    info = px.solver_info(pd)
    Lg, Ug = px.get_coeftab(pd, with_u=(fact == "GETRF"))
    rel = r.compare_panels(Lg, info, 0, mask_upper=(fact == "POTRF"))
    assert rel < tol, rel
    if fact == "GETRF":
        relu = r.compare_panels(Ug, info, 1)
        assert relu < tol, relu


@pytest.mark.parametrize("name,fact,magn,pivots", [("small", "SYTRF", 1e-14, 4997),
                                                    ("orsirr", "GETRF", 1e-3, 191),
                                                    ("orsirr", "GETRF", 0.0, 0)])
def test_fixture_on_reference_analysis(lib, ref_mod, name, fact, magn, pivots):
    A, _ = fixture_matrix(name)
    r = ref_mod.RefPastix(A, fact, nthreads=NTHREADS, magn_ctrl=magn)
    r.analyze(perm=_product_perm(A, fact))
    assert r.numfact() == pivots
    pd, S = _gpu_on_reference_structure(r, A, fact, magn)
    assert int(pd.iparm[px.iparm.static_pivoting]) == pivots
    _check_factors(r, pd, fact, 1e-12)


def _grid_case(name):
    if name == "lap100":
        return gen.laplacian7(100, 100, 100), (100, 100, 100), "POTRF", 1
    if name == "grf512":
        A, grid, fact = gen.workload("grf512")
        return A, grid, fact, 1
    if name == "cd32":
        return gen.convdiff27(32, 32, 32), (32, 32, 32), "GETRF", 1
    if name == "el24":
        K, _ = gen.elastic27_dof3(24, 24, 24)
        return K, (24, 24, 24), "SYTRF", 3
    raise KeyError(name)


# dof = 3: block sizes counted in nodes by the reference; 53..106 nodes keep
# the expanded widths within the GPU kernels' 384 columns, so that the product
# splits on the node symbol as the reference does
BLOCKSIZES = {"el24": (53, 106)}


@pytest.mark.parametrize("name", ["lap100", "grf512", "cd32", "el24"])
def test_grid_factors_match_reference(lib, ref_mod, name):
    A, grid, fact, dof = _grid_case(name)
    bmin, bmax = BLOCKSIZES.get(name, (None, None))
    r = ref_mod.RefPastix(A, fact, nthreads=NTHREADS, dof=dof, min_bs=bmin, max_bs=bmax)
    r.analyze(grid=grid)
    s = r.structure()
    pd, S, info = analyse(A, grid, fact, min_bs=bmin, max_bs=bmax)
    # the product's own analysis is the reference's
    assert np.array_equal(_expanded(s["permtab"], A.shape[0]), np.asarray(info["permtab"]))
    for k in ("cb_fcol", "cb_lcol", "cb_fblok", "bk_frow", "bk_lrow", "bk_fcblk"):
        assert np.array_equal(np.asarray(s[k]), np.asarray(info[k])), k
    npiv = r.numfact()
    px.task_numfact(pd, S)
    assert int(pd.iparm[px.iparm.static_pivoting]) == npiv
    _check_factors(r, pd, fact, 1e-11 if name == "el24" else 1e-12)


@pytest.mark.parametrize("name,fact", [("lap20", "POTRF"), ("cd64", "GETRF"), ("lap20", "SYTRF")])
def test_fp32_factors_match_reference_fp32(lib, ref_mod, name, fact):
    """IPARM_MIXED: both codes factor in FP32 (the reference with its s-precision
    kernels, the GPU with FP32 accumulation over split-BF16 tensor products)."""
    A, grid, _ = gen.workload(name, small=(name != "lap20"))
    r = ref_mod.RefPastix(A, fact, nthreads=NTHREADS, mixed=True)
    r.analyze(grid=grid)
    r.numfact()
    pd, S, info = analyse(A, grid, fact, mixed=True)
    px.task_numfact(pd, S)
    _check_factors(r, pd, fact, 2e-6)


@pytest.mark.parametrize("name,fact,refine,magn,mixed", [
    ("orsirr", "GETRF", 0, 0.0, False),    # GMRES (example/CTestLists.txt:121)
    ("orsirr", "GETRF", 3, 0.0, False),    # BiCGStab
    ("small", "SYTRF", 1, 1e-14, False),   # CG with magnitude control 1e-14 (:117, :147)
    ("orsirr", "GETRF", 0, 0.0, True),     # FP32 factors + FP64 GMRES (IPARM_MIXED)
])
def test_refinement_matches_reference(lib, ref_mod, name, fact, refine, magn, mixed):
    """pastix_task_solve + pastix_task_refine on the reference's own analysis:
    both reach the reference's stopping test ||b - Ax|| / ||b|| <= 1e-12
    (refinement/z_refine_gmres.c:164-172) and take the same number of Krylov
    iterations, within one (the factors agree to rounding, so the residual
    histories agree until the last digits)."""
    A, _ = fixture_matrix(name)
    r = ref_mod.RefPastix(A, fact, nthreads=NTHREADS, magn_ctrl=magn, mixed=mixed)
    r.iparm[ref_mod.IPARM_REFINEMENT] = refine
    r.dparm[ref_mod.DPARM_EPSILON_REFINEMENT] = 1e-12
    r.analyze(perm=_product_perm(A, fact))
    r.numfact()
    n = A.shape[0]
    rng = np.random.default_rng(9)
    b = A @ rng.uniform(-1, 1, n)
    xr = r.refine(b, r.solve(b))[:, 0]
    it_ref = int(r.iparm[ref_mod.IPARM_NBITER])

    s = r.structure()
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = FACT_ID[fact]
    ip[px.iparm.refinement] = refine
    ip[px.iparm.mixed] = 1 if mixed else 0
    dp[px.dparm.epsilon_magn_ctrl] = magn
    dp[px.dparm.epsilon_refinement] = 1e-12
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    px.set_symbol(pd, S, s["permtab"], s["cb_fcol"], s["cb_lcol"], s["cb_fblok"], s["bk_frow"], s["bk_lrow"],
                  s["bk_fcblk"])
    px.task_numfact(pd, S)
    x = b.copy()
    px.task_solve(pd, S, x)
    px.task_refine(pd, S, b, x)
    it_gpu = int(pd.iparm[px.iparm.nbiter])
    for xx in (xr, x):
        assert np.linalg.norm(b - A @ xx) <= 1e-12 * np.linalg.norm(b)
    assert abs(it_gpu - it_ref) <= 1, (it_gpu, it_ref)
