"""Shared fixtures: build the in-tree library and the oracle once per session."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from pastix_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    oracle.load()
    return oracle


FACT_ID = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}


def analyse(A, grid, fact, mixed=False, min_bs=None, max_bs=None):
    """Analysis through the C ABI with the grid ordering; returns (pd, spm, info)."""
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = FACT_ID[fact]
    if mixed:
        ip[px.iparm.mixed] = 1
    if min_bs:
        ip[px.iparm.min_blocksize] = min_bs
    if max_bs:
        ip[px.iparm.max_blocksize] = max_bs
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    px.analyze_grid(pd, S, *grid)
    return pd, S, px.solver_info(pd)


def backward_error(A, x, b) -> float:
    import scipy.sparse.linalg as spla
    r = b - A @ x
    return float(np.linalg.norm(r) / (spla.norm(A) * np.linalg.norm(x) + np.linalg.norm(b)))


@pytest.fixture(scope="session")
def ref_mod():
    """The reference PaStiX compiled from its sources (oracle/_ref).  Built here
    when the source tree is on this machine; the tests that need it are skipped
    when it is neither built nor buildable."""
    from oracle import ref
    if not ref.available():
        from oracle.refbuild import build_ref
        src = build_ref.ref_root()
        if not (src / "sopalin" / "pastix_task_sopalin.c").exists():
            pytest.skip("oracle/_ref is not built and the reference source tree is absent")
        ref.build(src)
    ref.load()
    return ref


def fixture_matrix(name):
    """A reference test matrix from tests/golden (CSC, 0-based) and its HB type."""
    import scipy.sparse as sps
    z = np.load(ROOT / "tests" / "golden" / f"{name}.npz")
    n = int(z["n"])
    A = sps.csc_matrix((z["values"], z["rowind"], z["colptr"]), shape=(n, n))
    if str(z["mxtype"])[1] == "S":  # symmetric: the file stores one triangle
        A = (A + sps.tril(A, -1).T).tocsc()
    return A, str(z["mxtype"])
