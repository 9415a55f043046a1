"""CPU pinning of the oracle.

No reference output vectors exist for this path (the reference's tests only
bound residuals), so the oracle is pinned by:
  * uniqueness: LL^T, LDL^T and LU without pivoting of a given permuted matrix
    are unique, so the oracle's factors must equal dense LAPACK / numpy
    factorizations of the same permuted matrix;
  * the reference's known-answer checks: backward error thresholds
    (example/simple.c:140), the SpMV bound of test/z_bcsc_tests.c:179-186,
    zero static pivots on SPD matrices, and convergence of the refinement on
    the reference's own fixtures (example/CTestLists.txt:117-149);
  * the static-pivot rule (kernels/core_zpotrfsp.c:80-83 and siblings)
    restated on a dense matrix.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sps

from conftest import ROOT, analyse, backward_error
from pastix_b200 import gen


def _dense_from_panels(info, P, lower_only=True):
    """Dense n x n lower-triangular image (diagonal included) of panel-layout coefficients."""
    n = int(info["n"])
    M = np.zeros((n, n))
    for k in range(int(info["cblknbr"])):
        fc = int(info["cb_fcol"][k])
        nc = int(info["cb_lcol"][k]) - fc + 1
        st = int(info["cb_stride"][k])
        base = int(info["cb_coef"][k])
        rows = np.concatenate([np.arange(info["bk_frow"][b], info["bk_lrow"][b] + 1)
                               for b in range(info["cb_fblok"][k], info["cb_fblok"][k + 1])])
        blk = P[base:base + st * nc].reshape(nc, st).T
        for c in range(nc):
            sel = rows >= fc + c if lower_only else np.ones_like(rows, bool)
            M[rows[sel], fc + c] = blk[sel, c]
    return M


def _ldl_nopiv(A):
    n = A.shape[0]
    W = A.copy()
    L = np.eye(n)
    d = np.zeros(n)
    for k in range(n):
        d[k] = W[k, k]
        L[k + 1:, k] = W[k + 1:, k] / d[k]
        W[k + 1:, k + 1:] -= np.outer(L[k + 1:, k], W[k, k + 1:])
    return L, d


def _lu_nopiv(A):
    n = A.shape[0]
    W = A.copy()
    for k in range(n):
        W[k + 1:, k] /= W[k, k]
        W[k + 1:, k + 1:] -= np.outer(W[k + 1:, k], W[k, k + 1:])
    return np.tril(W, -1) + np.eye(n), np.triu(W)


def test_potrf_equals_dense_cholesky(lib, oracle_mod):
    A = gen.laplacian7(8, 7, 6)
    pd, S, info = analyse(A, (8, 7, 6), "POTRF")
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, _, npiv = oracle_mod.factor(sym, Ap, "POTRF", oracle_mod.criterion(Ap))
    assert npiv == 0
    L = _dense_from_panels(info, oracle_mod.to_panels(sym, L2))
    Lref = np.linalg.cholesky(Ap.toarray())
    assert np.linalg.norm(L - Lref) <= 1e-13 * np.linalg.norm(Lref)


def test_sytrf_equals_dense_ldlt(lib, oracle_mod):
    A, grid, _ = gen.workload("el48", small=True)  # shifted indefinite, element growth ~1e3
    pd, S, info = analyse(A, grid, "SYTRF")
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, _, npiv = oracle_mod.factor(sym, Ap, "SYTRF", oracle_mod.criterion(Ap))
    M = _dense_from_panels(info, oracle_mod.to_panels(sym, L2))
    Lref, dref = _ldl_nopiv(Ap.toarray())
    Mref = np.tril(Lref, -1) + np.diag(dref)
    assert np.linalg.norm(M - Mref) <= 1e-11 * np.linalg.norm(Mref)


def test_getrf_equals_dense_lu(lib, oracle_mod):
    A = gen.convdiff27(7, 6, 5)
    pd, S, info = analyse(A, (7, 6, 5), "GETRF")
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, U2, npiv = oracle_mod.factor(sym, Ap, "GETRF", oracle_mod.criterion(Ap))
    Lref, Uref = _lu_nopiv(Ap.toarray())
    Ld = _dense_from_panels(info, oracle_mod.to_panels(sym, L2))   # L strictly below, U's diagonal on it
    Ud = _dense_from_panels(info, oracle_mod.to_panels(sym, U2))   # U^T (diagonal included)
    assert np.linalg.norm(np.tril(Ld, -1) - np.tril(Lref, -1)) <= 1e-12 * np.linalg.norm(Lref)
    assert np.linalg.norm(Ud.T - Uref) <= 1e-12 * np.linalg.norm(Uref)


@pytest.mark.parametrize("name,fact", [("lap20", "POTRF"), ("grf512", "POTRF"), ("cd64", "GETRF"), ("el48", "SYTRF")])
def test_oracle_solve_backward_error(lib, oracle_mod, name, fact):
    A, grid, _ = gen.workload(name, small=(name != "lap20"))
    pd, S, info = analyse(A, grid, fact)
    sym = oracle_mod.Symbol(info)
    Af = S.full()
    Ap = oracle_mod.permuted_full(Af, info["permtab"])
    L, U, npiv = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap))
    if name in ("lap20", "grf512"):
        assert npiv == 0  # SPD: no static pivot
    perm = info["permtab"]
    xt = gen.rhs_uniform(A.shape[0], 1, 0)[:, 0]
    b = Af @ xt
    bp = np.zeros_like(b)
    bp[perm] = b
    x = oracle_mod.solve(sym, fact, L, U, bp)[:, 0][perm]
    assert backward_error(Af, x, b) <= 1e-15


def test_static_pivot_rule_dense(lib, oracle_mod):
    """Dense restatement of the static-pivot rule (replace |d| < crit by +-crit,
    count): same count and same factor as the oracle on a forced threshold."""
    A = gen.laplacian7(6, 6, 6)
    pd, S, info = analyse(A, (6, 6, 6), "SYTRF")
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    crit = 5.5
    L2, _, npiv = oracle_mod.factor(sym, Ap, "SYTRF", crit)
    W = Ap.toarray()
    n = W.shape[0]
    cnt = 0
    Lr = np.eye(n)
    d = np.zeros(n)
    for k in range(n):
        dk = W[k, k]
        if abs(dk) < crit:
            dk = -crit if dk < 0 else crit
            cnt += 1
        d[k] = dk
        Lr[k + 1:, k] = W[k + 1:, k] / dk
        W[k + 1:, k + 1:] -= np.outer(Lr[k + 1:, k], W[k, k + 1:])
    assert cnt == npiv and cnt > 0
    M = _dense_from_panels(info, oracle_mod.to_panels(sym, L2))
    assert np.linalg.norm(M - (np.tril(Lr, -1) + np.diag(d))) <= 1e-12 * np.linalg.norm(M)


def test_spmv_bound(lib, oracle_mod):
    """test/z_bcsc_tests.c:179-186: ||y - y_ref||_inf / ((||A|| + ||x|| + ||y||) nnz/n eps) <= 10,
    for the permuted-CSR product the GPU SpMV restates (host reference here)."""
    A, grid, _ = gen.workload("cd64", small=True)
    pd, S, info = analyse(A, grid, "GETRF")
    perm = info["permtab"]
    Af = S.full()
    Ap = oracle_mod.permuted_full(Af, perm).tocsr()
    rng = np.random.default_rng(5)
    x = rng.uniform(-0.5, 0.5, A.shape[0])
    y = Af @ x
    xp = np.zeros_like(x)
    xp[perm] = x
    yp = np.zeros_like(y)
    for i in range(A.shape[0]):  # row products in CSR order
        s = 0.0
        for p in range(Ap.indptr[i], Ap.indptr[i + 1]):
            s += Ap.data[p] * xp[Ap.indices[p]]
        yp[i] = s
    err = np.abs(yp[perm] - y).max()
    nrm = np.abs(Af).sum(axis=0).max() + np.abs(x).max() + np.abs(y).max()
    assert err / (nrm * (A.nnz / A.shape[0]) * np.finfo(float).eps) <= 10


def _fixture(name):
    z = np.load(ROOT / "tests" / "golden" / f"{name}.npz")
    n = int(z["n"])
    return sps.csc_matrix((z["values"], z["rowind"], z["colptr"]), shape=(n, n))


def test_fixture_orsirr_lu_gmres(lib, oracle_mod):
    """orsirr.rua with LU + GMRES converges to 1e-12 (example/CTestLists.txt:121,148)."""
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    A = _fixture("orsirr")
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.LU
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General)
    px.task_analyze(pd, S)
    info = px.solver_info(pd)
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(A, info["permtab"])
    L, U, npiv = oracle_mod.factor(sym, Ap, "GETRF", oracle_mod.criterion(Ap))
    b = A @ np.ones(A.shape[0])
    perm = info["permtab"]
    bp = np.zeros_like(b)
    bp[perm] = b
    prec = lambda r: oracle_mod.solve(sym, "GETRF", L, U, r)[:, 0]  # noqa: E731
    x, it = oracle_mod.refine_gmres(Ap.tocsr(), bp, prec(bp), prec)
    assert np.linalg.norm(bp - Ap @ x) / np.linalg.norm(bp) <= 1e-12


def test_fixture_small_rsa_ldlt(lib, oracle_mod):
    """small.rsa with LDL^T, magnitude control 1e-14 and CG (example/CTestLists.txt:117,147)."""
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    A = _fixture("small")
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.LDLT
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.task_analyze(pd, S)
    info = px.solver_info(pd)
    sym = oracle_mod.Symbol(info)
    Af = S.full()
    Ap = oracle_mod.permuted_full(Af, info["permtab"])
    L, U, npiv = oracle_mod.factor(sym, Ap, "SYTRF", oracle_mod.criterion(Ap, 1e-14))
    b = Af @ np.ones(A.shape[0])
    perm = info["permtab"]
    bp = np.zeros_like(b)
    bp[perm] = b
    prec = lambda r: oracle_mod.solve(sym, "SYTRF", L, None, r)[:, 0]  # noqa: E731
    x, it = oracle_mod.refine_cg(Ap.tocsr(), bp, prec(bp), prec)
    assert np.linalg.norm(bp - Ap @ x) / np.linalg.norm(bp) <= 1e-12
