"""Refinement iterations of the reference PaStiX (oracle/_ref, built from its
sources) with FP64 factors and with FP32 factors (IPARM_MIXED), on one of the
benchmark workloads at full size: how many Krylov iterations the reference's
own mixed-precision path needs to reach the backward-error target
(DPARM_EPSILON_REFINEMENT), next to its FP64 path.  Test infrastructure: it
runs on the host only.

    python -m oracle.refbuild.refine_iters el48 [threads]
"""
from __future__ import annotations

import sys
import time

import numpy as np


def main(argv: list[str]) -> int:
    from oracle import ref as R
    from pastix_b200 import gen
    name = argv[1] if len(argv) > 1 else "el48"
    nthreads = int(argv[2]) if len(argv) > 2 else 8
    A, grid, fact = gen.workload(name)
    dof = 3 if name == "el48" else 1
    rng = np.random.default_rng(1)
    b = A @ rng.uniform(-1.0, 1.0, A.shape[0])
    refine = {"SYTRF": 0, "GETRF": 0, "POTRF": 1}[fact]  # GMRES, CG for LL^T (as the bench)
    for mixed in (False, True):
        r = R.RefPastix(A, fact, nthreads=nthreads, dof=dof, mixed=mixed)
        r.iparm[R.IPARM_REFINEMENT] = refine
        r.dparm[R.DPARM_EPSILON_REFINEMENT] = 1e-12
        r.analyze(grid=grid)
        t0 = time.perf_counter()
        r.numfact()
        t1 = time.perf_counter()
        x = r.refine(b, r.solve(b))[:, 0]
        t2 = time.perf_counter()
        res = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
        print(f"{name} {'FP32 factors (IPARM_MIXED)' if mixed else 'FP64 factors'}: "
              f"{int(r.iparm[R.IPARM_NBITER])} iterations, ||b - Ax|| / ||b|| = {res:.2e}, "
              f"factor {t1 - t0:.1f} s, solve + refine {t2 - t1:.1f} s ({nthreads} threads)", flush=True)
        r.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
