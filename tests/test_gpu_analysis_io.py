"""A system factorized and solved on the GPU from an analysis loaded from files
(IPARM_IO_STRATEGY = PastixIOLoad with the files a PastixIOSave run wrote):
the same solution as with the analysis computed in place."""
from __future__ import annotations

import glob
import os
import shutil

import numpy as np
import pytest

from conftest import backward_error
from pastix_b200 import gen
from pastix_b200 import pastix as px
from pastix_b200.spm import mtxtype, spmatrix

pytestmark = pytest.mark.gpu


def _solve(A, io, ordering=None):
    ip, dp = px.initParam()
    ip[px.iparm.io_strategy] = int(io)
    if ordering is not None:
        ip[px.iparm.ordering] = int(ordering)
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.task_analyze(pd, S)
    px.task_numfact(pd, S)
    xt = np.random.default_rng(4).uniform(-1, 1, A.shape[0])
    b = S.full() @ xt
    x = b.copy()
    px.task_solve(pd, S, x)
    return S.full(), b, x


def test_factor_and_solve_from_loaded_analysis(lib, tmp_path, monkeypatch):
    A = gen.laplacian7(14, 13, 12)
    monkeypatch.setenv("PASTIX_OUTPUT_DIR", str(tmp_path / "pastix"))
    monkeypatch.delenv("PASTIX_FILE_ORDER", raising=False)
    Af, b, x_ref = _solve(A, px.io.Save)
    d = glob.glob(str(tmp_path / "pastix-*"))[0]
    shutil.copy(os.path.join(d, "symbgen"), tmp_path / "symbname")
    monkeypatch.setenv("PASTIX_FILE_ORDER", os.path.join(d, "ordergen"))
    monkeypatch.chdir(tmp_path)
    _, _, x = _solve(A, px.io.Load, px.ordering.Personal)
    assert backward_error(Af, x, b) <= 1e-14
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) <= 1e-12
