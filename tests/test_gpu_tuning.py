"""Update-tile buckets (pgpu_set_tuning) and their autotuner (pgpu_autotune):
every bucket setting computes the same factors as the default one (FP64 to
1e-12, FP32 to FP32 rounding), and the autotuner leaves one of its candidates
in effect with the matrix factorized."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import analyse
from pastix_b200 import gen
from pastix_b200 import pastix as px

pytestmark = pytest.mark.gpu

TOL = {False: 1e-12, True: 2e-6}


def _case(fact):
    if fact == "GETRF":
        return gen.convdiff27(16, 16, 16), (16, 16, 16)
    return gen.laplacian7(24, 24, 24), (24, 24, 24)


def _used(info, fact):
    """Panel entries that hold factor values: for LL^T and LDL^T the strict
    upper triangle of each diagonal block is not part of the factor (the
    update tiles may leave anything there)."""
    keep = np.ones(max(1, int(info["coefnbr"])), dtype=bool)
    if fact == "GETRF":
        return keep
    for k in range(info["cblknbr"]):
        nc = int(info["cb_lcol"][k] - info["cb_fcol"][k] + 1)
        st = int(info["cb_stride"][k])
        base = int(info["cb_coef"][k])
        r, c = np.triu_indices(nc, 1)  # r < c: row r of column c (column major, ld = stride)
        keep[base + c * st + r] = False
    return keep


def _factors(pd, vals, fact, keep):
    px.numfact_device(pd, vals)
    L, U = px.get_coeftab(pd, with_u=(fact == "GETRF"))
    out = [L.astype(np.float64)[keep]] + ([U.astype(np.float64)[keep]] if U is not None else [])
    return out, int(pd.iparm[px.iparm.static_pivoting])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("fact,mixed", [("POTRF", False), ("SYTRF", False), ("GETRF", False),
                                        ("POTRF", True), ("GETRF", True)])
def test_buckets_give_same_factors(lib, fact, mixed):
    A, grid = _case(fact)
    pd, S, info = analyse(A, grid, fact, mixed=mixed)
    vals = torch.tensor(S.values, device="cuda")
    assert px.get_tuning(pd) == (32, 32, 32)
    keep = _used(info, fact)
    ref, npiv0 = _factors(pd, vals, fact, keep)
    settings = [(64, 32, 96)] if mixed else [(8, 16, 32), (1, 1, 32), (64, 32, 32)]
    if mixed:
        settings.append((32, 32, 48))
    for st in settings:
        px.set_tuning(pd, *st)
        assert px.get_tuning(pd) == st
        got, npiv = _factors(pd, vals, fact, keep)
        assert npiv == npiv0
        for g, r in zip(got, ref):
            assert _rel(g, r) <= TOL[mixed], (st, _rel(g, r))
    assert lib.pgpu_device_status(pd.ptr) == 0


@pytest.mark.parametrize("mixed", [False, True])
def test_autotune(lib, mixed):
    A, grid = _case("POTRF")
    pd, S, info = analyse(A, grid, "POTRF", mixed=mixed)
    pd.iparm[px.iparm.refinement] = px.refine.CG
    vals = torch.tensor(S.values, device="cuda")
    chosen = px.autotune(pd, vals)
    assert px.get_tuning(pd) == chosen
    if mixed:
        assert chosen[2] in (32, 48, 64, 96)
    else:
        assert chosen[0] in (8, 16, 32, 64) and chosen[1] in (16, 32)
    # factorized with the chosen buckets: a solve works without another numfact
    n = A.shape[0]
    xt = np.random.default_rng(1).uniform(-1, 1, n)
    b = torch.tensor(S.full() @ xt, device="cuda")
    x = torch.zeros_like(b)
    px.solve_refine_device(pd, b, x)
    assert np.linalg.norm(x.cpu().numpy() - xt) / np.linalg.norm(xt) < 1e-10

