"""CUDA-graph replay of the factorization and solve launch sequences
(pgpu_graphs) against kernel-by-kernel launches: same factors, same
static-pivot counts, same solutions and the same launch accounting, on the
capture call and on replays with new matrix values and a new static-pivot
threshold."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import analyse
from pastix_b200 import gen
from pastix_b200 import pastix as px

pytestmark = pytest.mark.gpu

# relative Frobenius; level updates scatter with atomics, so the last bits may
# differ between any two runs (graph or not)
TOL = {False: 1e-12, True: 2e-6}

CASES = [("POTRF", False), ("SYTRF", False), ("GETRF", False), ("POTRF", True), ("GETRF", True)]


def _case(fact):
    if fact == "GETRF":
        return gen.convdiff27(12, 12, 12), (12, 12, 12)
    return gen.laplacian7(14, 14, 14), (14, 14, 14)


def _factor(pd, vals, fact):
    px.numfact_device(pd, vals)
    L, U = px.get_coeftab(pd, with_u=(fact == "GETRF"))
    L = L.astype(np.float64)
    return L, (U.astype(np.float64) if U is not None else None), int(pd.iparm[px.iparm.static_pivoting])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("fact,mixed", CASES)
def test_graph_replay_matches_direct_launches(lib, fact, mixed):
    A, grid = _case(fact)
    pd, S, info = analyse(A, grid, fact, mixed=mixed)
    n = A.shape[0]
    v0 = torch.tensor(S.values, device="cuda")
    v1 = v0 * 1.75  # new values: new norm, new static-pivot threshold
    g = torch.Generator(device="cuda").manual_seed(3)
    B = (torch.rand(n, 2, dtype=torch.float64, device="cuda", generator=g) - 0.5).t().contiguous().t()

    px.graphs(pd, False)
    ref = []
    for v in (v0, v1):
        px.profile(pd, False)
        L, U, npiv = _factor(pd, v, fact)
        X = B.clone()
        px.solve_device(pd, X)
        cnt = {k: c for k, (_, c) in px.profile_get(pd).items()}
        ref.append((L, U, npiv, X, cnt))

    px.graphs(pd, True)
    # capture call, then replays; the second value set replays the same graph
    for v, (Lr, Ur, npr, Xr, cntr) in [(v0, ref[0]), (v0, ref[0]), (v1, ref[1]), (v0, ref[0])]:
        px.profile(pd, False)
        L, U, npiv = _factor(pd, v, fact)
        X = B.clone()
        px.solve_device(pd, X)
        torch.cuda.synchronize()
        cnt = {k: c for k, (_, c) in px.profile_get(pd).items()}
        assert npiv == npr
        assert _rel(L, Lr) <= TOL[mixed]
        if Ur is not None:
            assert _rel(U, Ur) <= TOL[mixed]
        assert (torch.linalg.norm(X - Xr) / torch.linalg.norm(Xr)).item() <= TOL[mixed]
        assert cnt == cntr
    assert lib.pgpu_device_status(pd.ptr) == 0


def test_graph_replay_new_threshold(lib):
    """The static-pivot threshold lives in device memory: a replay after the
    threshold changed replaces pivots with the new value."""
    A, grid = _case("POTRF")
    pd, S, info = analyse(A, grid, "POTRF")
    vals = torch.tensor(S.values, device="cuda")
    out = {}
    for graphs in (False, True):
        px.graphs(pd, graphs)
        for thr in (10.0, 20.0, 10.0):  # absolute thresholds above the diagonal (6.001)
            pd.dparm[px.dparm.epsilon_magn_ctrl] = -thr
            L, _, npiv = _factor(pd, vals, "POTRF")
            out.setdefault(thr, []).append((L, npiv))
    for thr, runs in out.items():
        L0, np0 = runs[0]
        assert np0 > 0
        for L, npiv in runs[1:]:
            assert npiv == np0
            assert _rel(L, L0) <= 1e-12
    assert _rel(out[10.0][0][0], out[20.0][0][0]) > 1e-3


def test_graph_refinement(lib):
    """FP32 factors + CG refinement with graphed solves reach 1e-12 as without graphs."""
    A, grid = _case("POTRF")
    pd, S, info = analyse(A, grid, "POTRF", mixed=True)
    pd.iparm[px.iparm.refinement] = px.refine.CG
    pd.dparm[px.dparm.epsilon_refinement] = 1e-12
    n = A.shape[0]
    vals = torch.tensor(S.values, device="cuda")
    xt = np.random.default_rng(5).uniform(-1, 1, n)
    b = torch.tensor(S.full() @ xt, device="cuda")
    res = {}
    for graphs in (False, True, True):
        px.graphs(pd, graphs)
        px.numfact_device(pd, vals)
        x = torch.zeros_like(b)
        px.solve_refine_device(pd, b, x)
        err = float(np.linalg.norm(x.cpu().numpy() - xt) / np.linalg.norm(xt))
        res.setdefault(graphs, []).append((err, int(pd.iparm[px.iparm.nbiter])))
    for runs in res.values():
        for err, it in runs:
            assert err < 1e-9
    assert abs(res[True][0][1] - res[False][0][1]) <= 1
