"""GPU checks of the remaining C entry points: the legacy one-call pastix(),
the numerical subtasks (applyorder / trsm / diag / solve), the transposed
solve, the device SpMV against SciPy, and the launch accounting."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import analyse, backward_error
from pastix_b200 import _lib, gen
from pastix_b200 import pastix as px
from pastix_b200._lib import PDBL, PINT
from pastix_b200.spm import mtxtype, spmatrix

pytestmark = pytest.mark.gpu


def test_legacy_pastix_one_call(lib):
    A = gen.laplacian7(10, 10, 10).tocsc()
    import scipy.sparse as sps
    L = sps.tril(A, format="csc")
    L.sort_indices()
    n = A.shape[0]
    colptr = (L.indptr + 1).astype(np.int64)          # Fortran numbering
    rowptr = (L.indices + 1).astype(np.int64)
    vals = L.data.astype(np.float64).copy()
    xt = np.random.default_rng(0).uniform(-1, 1, n)
    b = (A @ xt).astype(np.float64)
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.LLT
    ip[px.iparm.mtx_type] = 112
    p = C.c_void_p()
    perm = np.zeros(n, np.int64)
    invp = np.zeros(n, np.int64)
    rc = lib.pastix(C.byref(p), 0, n, colptr.ctypes.data_as(PINT), rowptr.ctypes.data_as(PINT),
                    vals.ctypes.data_as(C.c_void_p), perm.ctypes.data_as(PINT), invp.ctypes.data_as(PINT),
                    b.ctypes.data_as(C.c_void_p), 1, ip.ctypes.data_as(PINT), dp.ctypes.data_as(PDBL))
    assert rc == 0
    assert not p  # END_TASK = clean finalizes
    assert np.linalg.norm(b - xt) / np.linalg.norm(xt) < 1e-12
    assert sorted(perm.tolist()) == list(range(n))


@pytest.mark.parametrize("fact", ["POTRF", "SYTRF", "GETRF"])
def test_subtask_sequence(lib, fact):
    """applyorder -> trsm (L) -> diag -> trsm (L^T or U) -> applyorder, as
    pastix_subtask_solve_adv does (sopalin/pastix_task_solve.c:543-649)."""
    A = gen.laplacian7(12, 12, 12) if fact != "GETRF" else gen.convdiff27(10, 10, 10)
    grid = (12, 12, 12) if fact != "GETRF" else (10, 10, 10)
    pd, S, info = analyse(A, grid, fact)
    px.task_numfact(pd, S)
    Af = S.full()
    xt = np.random.default_rng(1).uniform(-1, 1, A.shape[0])
    b = np.asfortranarray(Af @ xt)
    l = _lib.load()
    bp = C.c_void_p()
    assert l.pastixRhsInit(C.byref(bp)) == 0
    n = A.shape[0]
    assert l.pastix_subtask_applyorder(pd.ptr, 391, n, 1, b.ctypes.data, n, bp) == 0
    if fact == "POTRF":
        assert l.pastix_subtask_trsm(pd.ptr, 141, 122, 111, 131, bp) == 0
        assert l.pastix_subtask_trsm(pd.ptr, 141, 122, 112, 131, bp) == 0
    elif fact == "SYTRF":
        assert l.pastix_subtask_trsm(pd.ptr, 141, 122, 111, 132, bp) == 0
        assert l.pastix_subtask_diag(pd.ptr, bp) == 0
        assert l.pastix_subtask_trsm(pd.ptr, 141, 122, 112, 132, bp) == 0
    else:
        assert l.pastix_subtask_trsm(pd.ptr, 141, 122, 111, 132, bp) == 0
        assert l.pastix_subtask_trsm(pd.ptr, 141, 121, 111, 131, bp) == 0
    x = np.zeros_like(b)
    assert l.pastix_subtask_applyorder(pd.ptr, 392, n, 1, x.ctypes.data, n, bp) == 0
    l.pastixRhsFinalize(bp)
    assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-10


def test_transposed_solve(lib):
    A, grid, _ = gen.workload("cd64", small=True)
    pd, S, info = analyse(A, grid, "GETRF")
    px.task_numfact(pd, S)
    Af = S.full()
    xt = np.random.default_rng(2).uniform(-1, 1, A.shape[0])
    b = np.asfortranarray(Af.T @ xt)
    pd.iparm[px.iparm.transpose_solve] = 112
    x = b.copy(order="F")
    px.task_solve(pd, S, x)
    assert backward_error(Af.T.tocsc(), x, b) < 1e-14


def test_device_spmv(lib):
    A, grid, _ = gen.workload("cd64", small=True)
    pd, S, info = analyse(A, grid, "GETRF")
    px.task_numfact(pd, S)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(A.shape[0])
    y = rng.standard_normal(A.shape[0])
    xd = torch.tensor(x, device="cuda")
    yd = torch.tensor(y, device="cuda")
    px.spmv_device(pd, 2.0, xd, -0.5, yd)
    torch.cuda.synchronize()
    ref = 2.0 * (S.full() @ x) - 0.5 * y
    assert np.linalg.norm(yd.cpu().numpy() - ref) <= 1e-13 * np.linalg.norm(ref)


def test_device_spmv_long_row(lib):
    """A row longer than the streamed SpMV's per-block capacity (an arrow
    matrix: one node coupled to every other) goes through the one-row blocks."""
    import scipy.sparse as sps
    n = 6000
    A = sps.lil_matrix((n, n))
    A.setdiag(4.0 * n)
    A[0, 1:] = 1.0
    A[1:, 0] = 1.0
    A = sps.csc_matrix(A)
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.POTRF
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.task_analyze(pd, S)
    px.task_numfact(pd, S)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    xd = torch.tensor(x, device="cuda")
    yd = torch.tensor(y, device="cuda")
    px.spmv_device(pd, 1.5, xd, 0.25, yd)
    torch.cuda.synchronize()
    ref = 1.5 * (A @ x) + 0.25 * y
    assert np.linalg.norm(yd.cpu().numpy() - ref) <= 1e-13 * np.linalg.norm(ref)


def test_static_pivots_counted(lib, oracle_mod):
    """A magnitude threshold above some pivots forces static pivoting
    (kernels/core_zpotrfsp.c:80-83); counts and factors match the oracle."""
    A = gen.laplacian7(10, 10, 10)
    pd, S, info = analyse(A, (10, 10, 10), "SYTRF")
    pd.dparm[px.dparm.epsilon_magn_ctrl] = -5.7  # absolute threshold
    px.task_numfact(pd, S)
    npiv = int(pd.iparm[px.iparm.static_pivoting])
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, _, npiv_o = oracle_mod.factor(sym, Ap, "SYTRF", 5.7)
    assert npiv == npiv_o and npiv > 0
    Lg, _ = px.get_coeftab(pd)
    Lo = oracle_mod.to_panels(sym, L2)
    assert np.linalg.norm(Lg - Lo) <= 1e-12 * np.linalg.norm(Lo)


def test_launch_accounting(lib):
    A = gen.laplacian7(16, 16, 16)
    pd, S, info = analyse(A, (16, 16, 16), "POTRF")
    px.task_numfact(pd, S)
    px.profile(pd, True)
    vals = torch.tensor(S.values, device="cuda")
    px.numfact_device(pd, vals)
    prof = px.profile_get(pd)
    px.profile(pd, False)
    assert prof["panel_small"][1] + prof["diag_large"][1] > 0
    assert sum(v[1] for v in prof.values()) >= info["nlevels"]
    assert all(v[0] >= 0 for v in prof.values())
