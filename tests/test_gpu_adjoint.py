"""Adjoint of the sparse solve (torch.autograd): gradients of
loss = 0.5 ||x - x_obs||^2, x = A(values)^{-1} b, with respect to b and to every
stored value of A, against central finite differences along 20 random
directions (relative error <= 1e-6) and against the gradient assembled from
the oracle's CPU solves (lambda = A^{-T} (x - x_obs), grad_a_ij = -lambda_i x_j).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from pastix_b200 import gen
from pastix_b200.autograd import SparseSolver, solve

pytestmark = pytest.mark.gpu

CASES = [("grf512", "POTRF"), ("cd64", "GETRF")]


def _setup(name, fact):
    A, grid, _ = gen.workload(name, small=True)
    solver = SparseSolver(A, fact, grid=grid)
    n = A.shape[0]
    rng = np.random.default_rng(7)
    vals = torch.tensor(solver.spm.values, device="cuda")
    b = torch.tensor(rng.standard_normal(n), device="cuda")
    x_obs = torch.tensor(rng.standard_normal(n), device="cuda")
    return A, solver, vals, b, x_obs


def _loss(solver, vals, b, x_obs):
    x = solve(vals, b, solver)
    return 0.5 * ((x - x_obs) ** 2).sum(), x


@pytest.mark.parametrize("name,fact", CASES)
def test_adjoint_vs_finite_differences(lib, name, fact):
    A, solver, vals, b, x_obs = _setup(name, fact)
    v = vals.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    loss, _ = _loss(solver, v, bb, x_obs)
    loss.backward()
    gv, gb = v.grad.clone(), bb.grad.clone()
    rng = np.random.default_rng(11)
    for _ in range(20):
        dv = torch.tensor(rng.standard_normal(vals.numel()), device="cuda") * vals.abs()
        db = torch.tensor(rng.standard_normal(b.numel()), device="cuda")
        h = 1e-6
        with torch.no_grad():
            fp, _ = _loss(solver, vals + h * dv, b + h * db, x_obs)
            fm, _ = _loss(solver, vals - h * dv, b - h * db, x_obs)
        fd = (fp - fm).item() / (2 * h)
        an = (gv * dv).sum().item() + (gb * db).sum().item()
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-300), (fd, an)


@pytest.mark.parametrize("name,fact", CASES)
def test_adjoint_vs_cpu_solves(lib, oracle_mod, name, fact):
    import scipy.sparse as sps
    A, solver, vals, b, x_obs = _setup(name, fact)
    v = vals.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    loss, x = _loss(solver, v, bb, x_obs)
    loss.backward()
    # CPU: oracle factorization of the same ordering, solves with A and A^T
    from pastix_b200 import pastix as px
    info = px.solver_info(solver.pd)
    sym = oracle_mod.Symbol(info)
    Af = solver.spm.full()
    Ap = oracle_mod.permuted_full(Af, info["permtab"])
    L, U, _ = oracle_mod.factor(sym, Ap, fact, oracle_mod.criterion(Ap))
    perm = info["permtab"]
    bh = b.cpu().numpy()
    bp = np.zeros_like(bh)
    bp[perm] = bh
    xc = oracle_mod.solve(sym, fact, L, U, bp)[:, 0][perm]
    g = xc - x_obs.cpu().numpy()
    gp = np.zeros_like(g)
    gp[perm] = g
    lam = oracle_mod.solve(sym, fact, L, U, gp, trans=True)[:, 0][perm]
    S = sps.coo_matrix(solver.spm.A)  # stored entries in spm order
    gvals = -lam[S.row] * xc[S.col]
    if fact != "GETRF":
        off = S.row != S.col
        gvals[off] -= lam[S.col[off]] * xc[S.row[off]]
    assert np.linalg.norm(bb.grad.cpu().numpy() - lam) <= 1e-10 * np.linalg.norm(lam)
    assert np.linalg.norm(v.grad.cpu().numpy() - gvals) <= 1e-10 * np.linalg.norm(gvals)


def test_backward_after_another_forward(lib):
    """Two forwards with different values on one solver, then the first
    backward: its gradient must be the one of its own matrix."""
    A, solver, vals, b, x_obs = _setup("grf512", "POTRF")
    v1 = vals.clone().requires_grad_(True)
    loss1, _ = _loss(solver, v1, b, x_obs)
    loss1.backward()
    g_ref = v1.grad.clone()

    v1 = vals.clone().requires_grad_(True)
    loss1, _ = _loss(solver, v1, b, x_obs)
    v2 = (vals * 1.5).requires_grad_(True)
    loss2, _ = _loss(solver, v2, b, x_obs)  # replaces the resident factors
    loss1.backward()
    assert torch.linalg.norm(v1.grad - g_ref) <= 1e-12 * torch.linalg.norm(g_ref)
    loss2.backward()
    assert torch.linalg.norm(v2.grad - g_ref) > 1e-3 * torch.linalg.norm(g_ref)
