"""GPU parity: the CUDA factorization and solve against the oracle, through the C ABI.

Bars: static-pivot counts equal; FP64 factors within 1e-12 relative Frobenius
of the oracle's (both stored in the same panel layout); solutions to backward
error <= 1e-14.  The shifted indefinite elastic matrix factored by LDL^T
without pivoting has element growth max|L| ~ 1.4e3: two CPU codes (the
reference and the oracle's restatement) already differ by up to 4e-12 on it,
so its bar is 1e-11.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import analyse, backward_error
from pastix_b200 import gen
from pastix_b200 import pastix as px

pytestmark = pytest.mark.gpu

CASES = [
    ("lap20", "POTRF", False),
    ("lap20", "SYTRF", False),
    ("grf512", "POTRF", True),
    ("cd64", "GETRF", True),
    ("el48", "SYTRF", True),
]
TOL = {"el48": 1e-11}


def _mask_compare(fact, info):
    """Entries that carry factor values (excludes the unused upper part of the
    diagonal blocks of POTRF, which holds update garbage in both codes)."""
    keep = np.ones(int(info["coefnbr"]), dtype=bool)
    if fact != "POTRF":
        return keep
    for k in range(int(info["cblknbr"])):
        nc = int(info["cb_lcol"][k] - info["cb_fcol"][k] + 1)
        st = int(info["cb_stride"][k])
        base = int(info["cb_coef"][k])
        for c in range(1, nc):
            keep[base + c * st: base + c * st + c] = False
    return keep


@pytest.mark.parametrize("name,fact,small", CASES)
def test_factor_parity(lib, oracle_mod, name, fact, small):
    A, grid, _ = gen.workload(name, small=small)
    pd, S, info = analyse(A, grid, fact)
    px.task_numfact(pd, S)
    Lg, Ug = px.get_coeftab(pd, with_u=(fact == "GETRF"))
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, U2, npiv = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap))
    Lo = oracle_mod.to_panels(sym, L2)
    assert int(pd.iparm[px.iparm.static_pivoting]) == npiv
    keep = _mask_compare(fact, info)
    rel = np.linalg.norm((Lg - Lo)[keep]) / np.linalg.norm(Lo[keep])
    assert rel < TOL.get(name, 1e-12), rel
    if fact == "GETRF":
        Uo = oracle_mod.to_panels(sym, U2)
        relu = np.linalg.norm(Ug - Uo) / np.linalg.norm(Uo)
        assert relu < 1e-12, relu


@pytest.mark.parametrize("name,fact,small", CASES)
@pytest.mark.parametrize("nrhs", [1, 5])
def test_solve(lib, name, fact, small, nrhs):
    A, grid, _ = gen.workload(name, small=small)
    pd, S, info = analyse(A, grid, fact)
    px.task_numfact(pd, S)
    Af = S.full()
    xt = gen.rhs_uniform(A.shape[0], nrhs, 0)
    b = np.asfortranarray(Af @ xt)
    x = b.copy(order="F")
    px.task_solve(pd, S, x)
    for j in range(nrhs):
        assert backward_error(Af, x[:, j], b[:, j]) < 1e-14


# FP32 factors (IPARM_MIXED): every update runs in FP32 (tcgen05 tiles with
# split BF16 terms for the big tasks, SIMT for the rest), so the factor must
# agree with the FP64 oracle to FP32 accuracy.  A BF16-only product would
# miss this bar by two orders of magnitude.
MIXED_CASES = [("lap20", "POTRF", False), ("cd64", "GETRF", True), ("lap20", "SYTRF", False)]


@pytest.mark.parametrize("name,fact,small", MIXED_CASES)
def test_fp32_factor_accuracy(lib, oracle_mod, name, fact, small):
    A, grid, _ = gen.workload(name, small=small)
    pd, S, info = analyse(A, grid, fact, mixed=True)
    px.task_numfact(pd, S)
    Lg, Ug = px.get_coeftab(pd, with_u=(fact == "GETRF"))
    assert Lg.dtype == np.float32
    sym = oracle_mod.Symbol(info)
    Ap = oracle_mod.permuted_full(S.full(), info["permtab"])
    L2, U2, npiv = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap))
    Lo = oracle_mod.to_panels(sym, L2)
    keep = _mask_compare(fact, info)
    rel = np.linalg.norm((Lg.astype(np.float64) - Lo)[keep]) / np.linalg.norm(Lo[keep])
    assert rel < 2e-6, rel
    if fact == "GETRF":
        Uo = oracle_mod.to_panels(sym, U2)
        relu = np.linalg.norm(Ug.astype(np.float64) - Uo) / np.linalg.norm(Uo)
        assert relu < 2e-6, relu
