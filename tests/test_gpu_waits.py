"""The kernels' spin waits are bounded: a wait that nothing satisfies gives up
and is reported, and the GPU context stays usable (pgpu_wait_selftest).  The
failure is made by a flag that nothing raises and an mbarrier phase that
nothing completes -- no fault, trap or endless loop."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from pastix_b200 import _lib

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_the_context_stays_usable(lib):
    out = (C.c_int * 2)()
    assert _lib.load().pgpu_wait_selftest(out) == 0
    assert list(out) == [1, 1]  # CTA 0: mbarrier wait, CTA 1: cluster-flag wait
    # the context still runs kernels: a factorization and solve afterwards
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    A = gen.laplacian7(12, 12, 12)
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.POTRF
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.analyze_grid(pd, S, 12, 12, 12)
    px.task_numfact(pd, S)
    b = A @ np.ones(A.shape[0])
    x = b.copy()
    px.task_solve(pd, S, x)
    assert np.linalg.norm(x - 1.0) < 1e-10 * np.sqrt(A.shape[0])
    assert _lib.load().pgpu_device_status(pd.ptr) == 0
