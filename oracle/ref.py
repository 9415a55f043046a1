"""The reference PaStiX itself, compiled from its sources -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of ``oracle/_ref/libpastix_ref.so`` (built by
``oracle/refbuild/build_ref.py`` where the reference source tree is present;
the built library travels with the repository's working copy).  It runs the
reference's own analysis (``pastix_subtask_order`` / ``symbfact`` /
``reordering`` / ``blend``), numerical factorization (``pastix_task_numfact``
with the scheduler chosen by IPARM_SCHEDULER), solve and refinement, and
exposes what the product must reproduce: the ordering, the SolverMatrix
structure, the factors, the static-pivot count.

Only the tests, ``__graft_entry__.smoke()`` and the reference arm of
``bench.py`` use it; the product never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import scipy.sparse as sps

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libpastix_ref.so"
I64P = C.POINTER(C.c_int64)
DP = C.POINTER(C.c_double)

# include/pastix/api.h indices used here
IPARM_VERBOSE = 0
IPARM_NNZEROS = 2
IPARM_MIN_BLOCKSIZE = 36
IPARM_MAX_BLOCKSIZE = 37
IPARM_FACTORIZATION = 43
IPARM_STATIC_PIVOTING = 45
IPARM_REFINEMENT = 51
IPARM_NBITER = 52
IPARM_ITERMAX = 53
IPARM_GMRES_IM = 54
IPARM_SCHEDULER = 55
IPARM_THREAD_NBR = 56
IPARM_MIXED = 71
IPARM_SIZE = 80
DPARM_EPSILON_REFINEMENT = 1
DPARM_RELATIVE_ERROR = 2
DPARM_EPSILON_MAGN_CTRL = 3
DPARM_FACT_TIME = 10
DPARM_FACT_THFLOPS = 12
DPARM_SOLV_TIME = 17
DPARM_REFINE_TIME = 22
DPARM_A_NORM = 23
DPARM_SIZE = 26

FACT = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}
SCHED = {"sequential": 0, "static": 1, "dynamic": 4}

_lib = None


def available() -> bool:
    return LIB.exists()


def build(src=None) -> Path:
    """Compile the reference (needs its source tree on this machine)."""
    from oracle.refbuild import build_ref
    return build_ref.build(Path(src) if src else None)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built (oracle/refbuild/build_ref.py)")
        from . import blas
        b = blas.find_openblas()
        if b is not None:
            for dep in blas.runtime_deps(b):
                try:
                    C.CDLL(str(dep), mode=C.RTLD_GLOBAL)
                except OSError:
                    pass
        lib = C.CDLL(str(LIB))
        lib.ref_new.restype = C.c_void_p
        lib.ref_iparm.restype = I64P
        lib.ref_iparm.argtypes = [C.c_void_p]
        lib.ref_dparm.restype = DP
        lib.ref_dparm.argtypes = [C.c_void_p]
        lib.ref_free.restype = None
        lib.ref_free.argtypes = [C.c_void_p]
        _lib = lib
    return _lib


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def symmetric_pattern(A) -> sps.csc_matrix:
    """A with the pattern of A + A^T (new entries explicit zeros), sorted CSC:
    what the reference's drivers hand to the analysis for an unsymmetric
    pattern (spmCheckAndCorrect)."""
    T = sps.coo_matrix(A)
    B = sps.coo_matrix((np.concatenate([T.data, np.zeros_like(T.data)]),
                        (np.concatenate([T.row, T.col]), np.concatenate([T.col, T.row]))),
                       shape=A.shape).tocsc()
    B.sum_duplicates()
    B.sort_indices()
    return B


def node_matrix(A, dof: int, lower: bool):
    """Scalar matrix A (dof unknowns per node, unknown v*dof+d of node v) as the
    SpM descriptor of a dof > 1 matrix: node CSC pattern, and per stored node
    pair (I, J) its dof x dof block A[I*dof:, J*dof:] column-major, as
    bcsc/bcsc_zinit.c reads it.  lower: keep the node pairs I >= J only."""
    T = sps.coo_matrix(A)
    n = A.shape[0] // dof
    r, c = T.row.astype(np.int64), T.col.astype(np.int64)
    P = sps.coo_matrix((np.ones(T.nnz), (r // dof, c // dof)), shape=(n, n)).tocsc()
    P.sum_duplicates()
    if lower:
        P = sps.tril(P, format="csc")
    P.sort_indices()
    # entry e of P has key col * n + row; keys are sorted because P is sorted CSC
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(P.indptr))
    keys = cols * n + P.indices.astype(np.int64)
    sel = (r // dof >= c // dof) if lower else np.ones(T.nnz, dtype=bool)
    k = (c[sel] // dof) * n + r[sel] // dof
    e = np.searchsorted(keys, k)
    vals = np.zeros(P.nnz * dof * dof)
    vals[e * dof * dof + (c[sel] % dof) * dof + r[sel] % dof] = T.data[sel]
    return P.indptr.astype(np.int64), P.indices.astype(np.int64), vals


class RefPastix:
    """One instance of the reference solver on one matrix.

    ``A``: SciPy sparse matrix; POTRF / SYTRF store its lower triangle
    (SpmSymmetric), GETRF the whole matrix with its pattern symmetrized by
    explicit zeros."""

    def __init__(self, A, fact: str = "POTRF", nthreads: int = 1, scheduler: str = "static",
                 magn_ctrl: float = 0.0, mixed: bool = False, min_bs: int | None = None,
                 max_bs: int | None = None, dof: int = 1):
        self.lib = load()
        self.fact = fact
        self.h = C.c_void_p(self.lib.ref_new())
        ip, dp = self.iparm, self.dparm
        ip[IPARM_FACTORIZATION] = FACT[fact]
        ip[IPARM_SCHEDULER] = SCHED[scheduler]
        ip[IPARM_THREAD_NBR] = int(nthreads)
        ip[IPARM_MIXED] = 1 if mixed else 0
        if min_bs:
            ip[IPARM_MIN_BLOCKSIZE] = min_bs
        if max_bs:
            ip[IPARM_MAX_BLOCKSIZE] = max_bs
        dp[DPARM_EPSILON_MAGN_CTRL] = magn_ctrl
        rc = self.lib.ref_init(self.h)
        if rc:
            raise RuntimeError(f"pastixInit failed ({rc})")
        A = sps.csc_matrix(A, dtype=np.float64)
        A.sum_duplicates()
        mtx = 111 if fact == "GETRF" else 112
        self.n = A.shape[0]
        if dof > 1:  # node descriptor with dof x dof blocks
            cp, ri, va = node_matrix(symmetric_pattern(A) if fact == "GETRF" else A, dof, lower=fact != "GETRF")
            self._cp, self._ri, self._va = _i64(cp), _i64(ri), np.ascontiguousarray(va)
            nn = self.n // dof
        else:
            if fact == "GETRF":
                A = symmetric_pattern(A)
            else:
                A = sps.tril(A, format="csc")
            A.sort_indices()
            self._cp, self._ri = _i64(A.indptr), _i64(A.indices)
            self._va = np.ascontiguousarray(A.data, dtype=np.float64)
            nn = self.n
        rc = self.lib.ref_set_matrix(self.h, C.c_int64(nn), self._cp.ctypes.data_as(I64P),
                                     self._ri.ctypes.data_as(I64P), self._va.ctypes.data_as(DP),
                                     C.c_int(mtx), C.c_int64(dof))
        if rc:
            raise RuntimeError(f"ref_set_matrix failed ({rc})")
        self._structure = None

    # parameter arrays (live views)
    @property
    def iparm(self):
        return np.ctypeslib.as_array(self.lib.ref_iparm(self.h), shape=(IPARM_SIZE,))

    @property
    def dparm(self):
        return np.ctypeslib.as_array(self.lib.ref_dparm(self.h), shape=(DPARM_SIZE,))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def analyze(self, grid=None, perm=None) -> None:
        nx, ny, nz = grid if grid is not None else (0, 0, 0)
        p = _i64(perm) if perm is not None else None
        rc = self.lib.ref_analyze(self.h, C.c_int64(nx), C.c_int64(ny), C.c_int64(nz),
                                  p.ctypes.data_as(I64P) if p is not None else None)
        if rc:
            raise RuntimeError(f"reference analysis failed ({rc})")
        self._structure = None

    def structure(self) -> dict:
        """Ordering + SolverMatrix, in the field names of the product's pgpu_solver_info."""
        if self._structure is not None:
            return self._structure
        sz = np.zeros(6, dtype=np.int64)
        self.lib.ref_sizes(self.h, sz.ctypes.data_as(I64P))
        n, cb, bk, coefnbr, ocb, on = (int(x) for x in sz)
        perm, peri = np.zeros(on, np.int64), np.zeros(on, np.int64)
        rang, tree = np.zeros(ocb + 1, np.int64), np.zeros(max(1, ocb), np.int64)
        self.lib.ref_get_order(self.h, *(a.ctypes.data_as(I64P) for a in (perm, peri, rang, tree)))
        arrs = {k: np.zeros(cb + 1 if k == "cb_fblok" else cb, np.int64)
                for k in ("cb_fcol", "cb_lcol", "cb_fblok", "cb_stride", "cb_type")}
        arrs.update({k: np.zeros(bk, np.int64) for k in ("bk_frow", "bk_lrow", "bk_fcblk")})
        self.lib.ref_get_solver(self.h, *(arrs[k].ctypes.data_as(I64P) for k in
                                          ("cb_fcol", "cb_lcol", "cb_fblok", "cb_stride", "cb_type",
                                           "bk_frow", "bk_lrow", "bk_fcblk")))
        s = dict(n=n, cblknbr=cb, bloknbr=bk, coefnbr=coefnbr, permtab=perm, peritab=peri,
                 rangtab=rang, treetab=tree[:ocb], thflops=float(self.dparm[DPARM_FACT_THFLOPS]), **arrs)
        self._structure = s
        return s

    def numfact(self) -> int:
        """pastix_task_numfact; returns the static-pivot count."""
        rc = self.lib.ref_numfact(self.h)
        if rc:
            raise RuntimeError(f"pastix_task_numfact failed ({rc})")
        return int(self.iparm[IPARM_STATIC_PIVOTING])

    def coef(self, coefind: np.ndarray, coefnbr: int, side: int = 0) -> np.ndarray:
        """Factors in the per-blok layout given by ``coefind`` (oracle.ora_layout)."""
        out = np.zeros(max(1, coefnbr), dtype=np.float64)
        ci = _i64(coefind)
        rc = self.lib.ref_get_coef(self.h, C.c_int(side), ci.ctypes.data_as(I64P), out.ctypes.data_as(DP))
        if rc:
            raise RuntimeError("ref_get_coef failed")
        return out

    def compare_panels(self, P: np.ndarray, info: dict, side: int = 0, mask_upper: bool = False) -> float:
        """Relative Frobenius distance between the reference's factors and
        factors P in the product's panel layout (``info``: pgpu_solver_info of
        the same structure), computed without a second copy of the factors."""
        P = np.ascontiguousarray(P)
        arrs = [_i64(info[k]) for k in ("cb_coef", "cb_stride", "bk_rowoff")]
        out = np.zeros(2)
        rc = self.lib.ref_compare_panels(self.h, C.c_int(side), P.ctypes.data_as(C.c_void_p),
                                         C.c_int(int(P.dtype == np.float32)),
                                         *(a.ctypes.data_as(I64P) for a in arrs), C.c_int(int(mask_upper)),
                                         out.ctypes.data_as(DP))
        if rc:
            raise RuntimeError("ref_compare_panels failed")
        return float(np.sqrt(out[0] / out[1]))

    def solve(self, B: np.ndarray) -> np.ndarray:
        X = np.asfortranarray(np.array(B, dtype=np.float64, copy=True))
        if X.ndim == 1:
            X = X.reshape(-1, 1, order="F")
        rc = self.lib.ref_solve(self.h, C.c_int64(X.shape[1]), X.ctypes.data_as(DP), C.c_int64(X.shape[0]))
        if rc:
            raise RuntimeError(f"pastix_task_solve failed ({rc})")
        return X

    def refine(self, B: np.ndarray, X: np.ndarray) -> np.ndarray:
        Bc = np.asfortranarray(np.array(B, dtype=np.float64, copy=True)).reshape(self.n, -1, order="F")
        Xc = np.asfortranarray(np.array(X, dtype=np.float64, copy=True)).reshape(self.n, -1, order="F")
        rc = self.lib.ref_refine(self.h, C.c_int64(Xc.shape[1]), Bc.ctypes.data_as(DP), C.c_int64(self.n),
                                 Xc.ctypes.data_as(DP), C.c_int64(self.n))
        if rc:
            raise RuntimeError(f"pastix_task_refine failed ({rc})")
        return Xc
