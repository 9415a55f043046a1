"""CPU checks of the host analysis: grid nested dissection, block symbolic
factorization, supernode splitting, flop count and level schedule."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import analyse
from pastix_b200 import gen
from pastix_b200 import pastix as px


def test_order_grid_known_answer(lib):
    """7x7x7 cube: the first cut is the plane x = 3 (ties prefer x), numbered
    last with y outer / z inner and decreasing numbers (order/order_grids.c:189-210)."""
    perm, peri, rang, tree = px.orderGrid(7, 7, 7)
    n = 343
    assert sorted(perm.tolist()) == list(range(n))
    assert np.array_equal(peri[perm], np.arange(n))
    assert rang[0] == 0 and rang[-1] == n and np.all(np.diff(rang) > 0)
    assert rang[-1] - rang[-2] == 49
    expect = [3 + 7 * (y + 7 * z) for y in range(7) for z in range(7)]  # numbers n-1, n-2, ...
    assert [int(peri[n - 1 - i]) for i in range(49)] == expect
    assert tree[-1] == -1
    assert np.all(tree[:-1] > np.arange(len(tree) - 1))
    # both halves have the cut plane as father
    top = len(tree) - 1
    assert (tree == top).sum() == 2


def test_order_grid_leaves():
    perm, peri, rang, tree = px.orderGrid(20, 20, 20)
    w = np.diff(rang)
    assert w.max() == 400  # the first separator plane
    # every leaf box has fewer than 15 vertices (order_grids.c:190)
    sons = np.bincount(tree[tree >= 0], minlength=len(tree))
    assert np.all(w[sons == 0] < 15)


def _struct_L(Ap):
    """Structural pattern of the Cholesky factor (column sets), by symbolic elimination."""
    n = Ap.shape[0]
    Ap = Ap.tocsc()
    cols = [set(Ap.indices[Ap.indptr[j]:Ap.indptr[j + 1]][Ap.indices[Ap.indptr[j]:Ap.indptr[j + 1]] > j])
            for j in range(n)]
    parent = [-1] * n
    for j in range(n):
        if cols[j]:
            p = min(cols[j])
            parent[j] = p
            cols[p] |= {r for r in cols[j] if r > p}
    return cols


@pytest.mark.parametrize("grid", [(6, 5, 4), (9, 9, 1), (5, 7, 6)])
def test_symbolic_structure_is_exact(lib, oracle_mod, grid):
    A = gen.laplacian7(*grid)
    pd, S, info = analyse(A, grid, "POTRF")
    Ap = oracle_mod.permuted_full(A, info["permtab"])
    cols = _struct_L(Ap)
    for k in range(info["cblknbr"]):
        f, l = info["cb_fcol"][k], info["cb_lcol"][k]
        rows = set()
        for b in range(info["cb_fblok"][k] + 1, info["cb_fblok"][k + 1]):
            rows |= set(range(info["bk_frow"][b], info["bk_lrow"][b] + 1))
        true = set()
        for c in range(f, l + 1):
            true |= {r for r in cols[c] if r > l}
        assert rows == true, k
        # bloks are maximal runs inside one facing cblk
        for b in range(info["cb_fblok"][k] + 1, info["cb_fblok"][k + 1] - 1):
            adj = info["bk_lrow"][b] + 1 == info["bk_frow"][b + 1]
            assert not (adj and info["bk_fcblk"][b] == info["bk_fcblk"][b + 1])


def test_split_widths(lib):
    A = gen.laplacian7(12, 12, 12)
    pd, S, info = analyse(A, (12, 12, 12), "POTRF", min_bs=6, max_bs=12)
    w = info["cb_lcol"] - info["cb_fcol"] + 1
    assert w.max() <= 12
    # the 144-column top separator was cut into pieces of 6..12 columns
    top = np.where(info["cb_lcol"] == 12 ** 3 - 1)[0][0]
    assert 6 <= w[top] <= 12
    # every piece of the split top separator carries one dense blok facing each later piece
    pieces = [k for k in range(info["cblknbr"]) if info["cb_fcol"][k] >= 12 ** 3 - 144]
    for i, k in enumerate(pieces):
        fb = info["cb_fblok"][k]
        faced = list(info["bk_fcblk"][fb + 1: fb + len(pieces) - i])
        assert faced == pieces[i + 1:]


def _sum1d(info, fact):
    """Independent restatement of pastixSymbolGetFlops / sum1d (symbol/symbol_cost.c:53-88)."""
    tot = 0.0
    for k in range(info["cblknbr"]):
        N = float(info["cb_lcol"][k] - info["cb_fcol"][k] + 1)
        M = float(sum(info["bk_lrow"][b] - info["bk_frow"][b] + 1
                      for b in range(info["cb_fblok"][k] + 1, info["cb_fblok"][k + 1])))
        if fact == "POTRF":
            f = N * ((N / 6 + 0.5) * N + 1 / 3) + N * ((N / 6) * N - 1 / 6)
            if M > 0:
                f += M * N * (N + 1) + N * M * (M + 1)
        elif fact == "GETRF":
            mu = 0.5 * N * (N * (N - N / 3 - 1) + N) + 2 / 3 * N
            ad = 0.5 * N * (N * (N - N / 3) - N) + N / 6
            f = mu + ad
            if M > 0:
                f += 2 * M * N * (N + 1) + 2 * M * M * N
        else:
            f = N * ((N / 6 + 0.5) * N + 10 / 3) + N * ((N / 6) * N - 1 / 6)
            if M > 0:
                f += M * N * (N + 1) + N * M + N * M * (M + 1) + M * M
        tot += f
    return tot


@pytest.mark.parametrize("fact", ["POTRF", "GETRF", "SYTRF"])
def test_flops(lib, fact):
    A = gen.laplacian7(10, 10, 10)
    pd, S, info = analyse(A, (10, 10, 10), fact)
    assert info["thflops"] == pytest.approx(_sum1d(info, fact), rel=1e-12)
    assert pd.dparm[px.dparm.fact_thflops] == pytest.approx(info["thflops"])


def test_levels_respect_dependencies(lib):
    A = gen.laplacian7(16, 16, 16)
    pd, S, info = analyse(A, (16, 16, 16), "POTRF")
    lvl = info["cb_level"]
    src = np.repeat(np.arange(info["cblknbr"]), np.diff(info["cb_fblok"]))
    off = info["bk_fcblk"] != src
    assert np.all(lvl[info["bk_fcblk"][off]] > lvl[src[off]])
    assert info["nlevels"] == lvl.max() + 1


def test_dof_expansion(lib):
    A, grid, fact = gen.workload("el48", small=True)  # 8^3 nodes x 3 unknowns
    pd, S, info = analyse(A, grid, fact)
    assert info["n"] == 3 * 8 ** 3
    w = info["cb_lcol"] - info["cb_fcol"] + 1
    assert np.all(w % 3 == 0)  # supernodes hold whole nodes
    perm = info["permtab"]
    assert np.all(perm[0::3] % 3 == 0) and np.all(perm[1::3] == perm[0::3] + 1)


def test_builtin_ordering_on_fixture(lib):
    """Matrices without a grid use the built-in nested dissection + supernode
    detection (stand-in for Scotch/Metis)."""
    import scipy.sparse as sps
    from conftest import ROOT
    from pastix_b200.spm import mtxtype, spmatrix
    z = np.load(ROOT / "tests" / "golden" / "orsirr.npz")
    n = int(z["n"])
    A = sps.csc_matrix((z["values"], z["rowind"], z["colptr"]), shape=(n, n))
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.LU
    pd = px.init(ip, dp)
    px.task_analyze(pd, spmatrix(A, mtxtype.General))
    info = px.solver_info(pd)
    assert info["n"] == n and info["cblknbr"] > 1
    assert sorted(info["permtab"].tolist()) == list(range(n))


def test_import_external_symbol(lib):
    """pgpu_set_symbol takes the structure of an analysis made elsewhere; the
    resulting solver layout equals the one from the library's own analysis."""
    A = gen.laplacian7(9, 8, 7)
    pd, S, info = analyse(A, (9, 8, 7), "POTRF")
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.POTRF
    pd2 = px.init(ip, dp)
    px.set_symbol(pd2, S, info["permtab"], info["cb_fcol"], info["cb_lcol"], info["cb_fblok"][:-1],
                  info["bk_frow"], info["bk_lrow"], info["bk_fcblk"])
    info2 = px.solver_info(pd2)
    for key in ("cb_fcol", "cb_lcol", "cb_fblok", "cb_stride", "cb_coef", "bk_frow", "bk_lrow", "bk_fcblk",
                "bk_rowoff", "permtab", "cb_level"):
        assert np.array_equal(info[key], info2[key]), key
    assert info2["thflops"] == info["thflops"]
    # a structure that misses a facing cblk is rejected
    bad = info["bk_fcblk"].copy()
    bad[info["cb_fblok"][0] + 1] = 0
    with pytest.raises(px.PastixError):
        px.set_symbol(pd2, S, info["permtab"], info["cb_fcol"], info["cb_lcol"], info["cb_fblok"][:-1],
                      info["bk_frow"], info["bk_lrow"], bad)
