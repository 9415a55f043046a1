"""Parity with the reference PaStiX itself, compiled from its sources
(oracle/_ref, oracle/refbuild/build_ref.py).  Host only.

1. The product's analysis (grid nested dissection, supernodes, level order,
   row reordering, symbolic factorization, split) produces exactly the
   reference's ordering and SolverMatrix structure: permutation, cblk column
   ranges, bloks and their facing cblks, and the flop count
   (pastix_task_analyze, blend/pastix_task_analyze.c:53).
2. The oracle's C restatement of the numerical factorization, run on the
   reference's own structure, reproduces the reference's factors (1e-13
   relative Frobenius, FP64) and static-pivot counts exactly -- including the
   reference's LDL^T test of small.rsa with magnitude control 1e-14
   (example/CTestLists.txt:117: 4997 static pivots) and an LU of orsirr.rua
   with a threshold large enough to make the sign-keeping replacement of
   kernels/core_zgetrfsp.c:81-89 fire.
These pin the oracle that the GPU parity tests use.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import analyse, fixture_matrix
from pastix_b200 import gen

STRUCT_KEYS = ("cb_fcol", "cb_lcol", "cb_fblok", "cb_stride", "bk_frow", "bk_lrow", "bk_fcblk")


def _dof(name):
    return 3 if name == "el48" else 1


def _expanded_perm(s, dof):
    p = np.asarray(s["permtab"])
    return p if dof == 1 else (p[:, None] * dof + np.arange(dof)).ravel()


@pytest.mark.parametrize("name", ["lap20", "grf512", "cd64", "el48"])
def test_analysis_identical_to_reference(lib, ref_mod, name):
    A, grid, fact = gen.workload(name, small=(name != "lap20"))
    r = ref_mod.RefPastix(A, fact, dof=_dof(name))
    r.analyze(grid=grid)
    s = r.structure()
    pd, S, info = analyse(A, grid, fact)
    assert (s["cblknbr"], s["bloknbr"], s["coefnbr"]) == (info["cblknbr"], info["bloknbr"], info["coefnbr"])
    assert np.array_equal(_expanded_perm(s, _dof(name)), np.asarray(info["permtab"]))
    for k in STRUCT_KEYS:
        assert np.array_equal(np.asarray(s[k]), np.asarray(info[k])), k
    assert s["thflops"] == info["thflops"]


# FP64 factors, relative Frobenius.  The shifted indefinite elastic matrix
# (LDL^T without pivoting, element growth ~1.4e3) amplifies the rounding of
# the two codes' different summation orders (the reference's blocked BLAS
# against plain loops) to a few 1e-12.
TOL = {"el48": 5e-12}


def test_analysis_identical_dof3_split(lib, ref_mod):
    """dof = 3: the reference splits the supernodes of the node symbol, widths
    in nodes.  With IPARM_MAX_BLOCKSIZE * dof within the GPU kernels' limit
    the product does the same, and both give one structure."""
    K, _ = gen.elastic27_dof3(16, 16, 16)
    grid = (16, 16, 16)
    r = ref_mod.RefPastix(K, "SYTRF", dof=3, min_bs=53, max_bs=106)
    r.analyze(grid=grid)
    s = r.structure()
    pd, S, info = analyse(K, grid, "SYTRF", min_bs=53, max_bs=106)
    assert s["cblknbr"] > 16 ** 3 // 106  # wide supernodes were split
    assert np.array_equal(_expanded_perm(s, 3), np.asarray(info["permtab"]))
    for k in STRUCT_KEYS:
        assert np.array_equal(np.asarray(s[k]), np.asarray(info[k])), k
    assert s["thflops"] == info["thflops"]


def _compare_factors(ref_mod, oracle_mod, r, A, fact, magn=0.0, tol=1e-13):
    s = r.structure()
    npiv_ref = r.numfact()
    sym = oracle_mod.Symbol(s)
    Afull = ref_mod.symmetric_pattern(A) if fact == "GETRF" else A
    Ap = oracle_mod.permuted_full(Afull, _perm_for(s, r.n))
    L, U, npiv = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap, magn))
    Lr = r.coef(sym.coefind, sym.coefnbr, 0)
    assert npiv == npiv_ref
    assert np.linalg.norm(Lr - L) <= tol * np.linalg.norm(L)
    if fact == "GETRF":
        Ur = r.coef(sym.coefind, sym.coefnbr, 1)
        assert np.linalg.norm(Ur - U) <= tol * np.linalg.norm(U)
    return npiv


def _perm_for(s, n):
    p = np.asarray(s["permtab"])
    dof = n // p.size
    return p if dof == 1 else (p[:, None] * dof + np.arange(dof)).ravel()


@pytest.mark.parametrize("name,fact", [("lap20", "POTRF"), ("lap20", "SYTRF"), ("cd64", "GETRF"),
                                       ("el48", "SYTRF"), ("grf512", "POTRF")])
def test_oracle_matches_reference_factors(ref_mod, oracle_mod, name, fact):
    A, grid, _ = gen.workload(name, small=(name != "lap20"))
    r = ref_mod.RefPastix(A, fact, nthreads=2, dof=_dof(name))
    r.analyze(grid=grid)
    assert _compare_factors(ref_mod, oracle_mod, r, A, fact, tol=TOL.get(name, 1e-13)) == 0


def _product_perm(A, fact):
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}[fact]
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    px.task_analyze(pd, S)
    return np.asarray(px.solver_info(pd)["permtab"]).copy()


def test_small_rsa_static_pivots(lib, ref_mod, oracle_mod):
    """The reference's LDL^T integration test of small.rsa: magnitude control
    1e-14 (example/CTestLists.txt:117).  The fixture has no grid: the
    reference is given a nested-dissection permutation and finds its
    supernodes itself (orderFindSupernodes + orderAmalgamate)."""
    A, mx = fixture_matrix("small")
    assert mx == "RSA"
    r = ref_mod.RefPastix(A, "SYTRF", nthreads=2, magn_ctrl=1e-14)
    r.analyze(perm=_product_perm(A, "SYTRF"))
    assert _compare_factors(ref_mod, oracle_mod, r, A, "SYTRF", 1e-14) == 4997


@pytest.mark.parametrize("magn,expected", [(0.0, 0), (1e-3, 191)])
def test_orsirr_lu_sign_keeping_pivots(lib, ref_mod, oracle_mod, magn, expected):
    """LU of orsirr.rua; with the threshold 1e-3 * ||A||_F the static pivots of
    kernels/core_zgetrfsp.c:81-89 (replacement keeping the sign) fire."""
    A, mx = fixture_matrix("orsirr")
    assert mx == "RUA"
    r = ref_mod.RefPastix(A, "GETRF", nthreads=2, magn_ctrl=magn)
    r.analyze(perm=_product_perm(A, "GETRF"))
    assert _compare_factors(ref_mod, oracle_mod, r, A, "GETRF", magn) == expected


def test_panel_comparison_helper(lib, ref_mod, oracle_mod):
    """ref_compare_panels (used by the GPU parity tests on full-size factors)
    against a plain comparison: the oracle's factors moved to the product's
    panel layout are at rounding distance, a planted error is seen."""
    A, grid, fact = gen.workload("lap20")
    r = ref_mod.RefPastix(A, fact, nthreads=2)
    r.analyze(grid=grid)
    r.numfact()
    pd, S, info = analyse(A, grid, fact)
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(A, np.asarray(info["permtab"]))
    L, _, _ = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap))
    P = oracle_mod.to_panels(sym, L)
    assert r.compare_panels(P, info, mask_upper=True) < 1e-14
    k = int(info["cblknbr"]) - 1  # last cblk: its diagonal entry
    P[int(info["cb_coef"][k])] *= 1.0 + 1e-6
    assert r.compare_panels(P, info, mask_upper=True) > 1e-9
