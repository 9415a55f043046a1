"""Python side of the oracle -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of ``oracle/_build/liboracle.so`` (the CPU restatement of
PaStiX's numerical factorization and solve, see oracle.c) plus a numpy
restatement of the refinement drivers
(refinement/z_refine_gmres.c:49, z_refine_grad.c:49, z_refine_bicgstab.c:49,
z_refine_pivot.c:48).  Only the tests, ``__graft_entry__.smoke()`` and the CPU
baseline of ``bench.py`` use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np
import scipy.sparse as sps

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
I64P = C.POINTER(C.c_int64)



class ora_symbol_t(C.Structure):
    _fields_ = [("n", C.c_int64), ("cblknbr", C.c_int64), ("bloknbr", C.c_int64),
                ("cb_fcol", I64P), ("cb_lcol", I64P), ("cb_fblok", I64P),
                ("bk_frow", I64P), ("bk_lrow", I64P), ("bk_fcblk", I64P)]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (idempotent)."""
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        lib.ora_layout.restype = C.c_int64
        lib.ora_factor.restype = C.c_int64
        lib.ora_factor.argtypes = [C.c_void_p, I64P, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        lib.ora_fill_d.restype = C.c_int
        lib.ora_fill_s.restype = C.c_int
        lib.ora_load_blas.restype = C.c_int
        lib.ora_load_blas.argtypes = [C.c_char_p]
        _lib = lib
    return _lib


def use_blas(enable: bool = True) -> bool:
    """Bind OpenBLAS for the GEMMs (CPU baseline timing); False when absent."""
    lib = load()
    if not enable:
        lib.ora_unload_blas()
        return False
    from . import blas
    for p in blas.candidates():
        # the wheel's OpenBLAS needs its bundled gfortran / quadmath, loaded globally first
        for dep in blas.runtime_deps(p):
            try:
                C.CDLL(str(dep), mode=C.RTLD_GLOBAL)
            except OSError:
                pass
        if lib.ora_load_blas(str(p).encode()) == 0:
            return True
    return False


FACT = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}


class Symbol:
    """The block symbolic structure (from the product's analysis) in oracle form."""

    def __init__(self, info: dict):
        self.info = info
        self.n = int(info["n"])
        self.cblknbr = int(info["cblknbr"])
        self.bloknbr = int(info["bloknbr"])
        self._arrs = [np.ascontiguousarray(info[k], dtype=np.int64) for k in
                      ("cb_fcol", "cb_lcol", "cb_fblok", "bk_frow", "bk_lrow", "bk_fcblk")]
        s = ora_symbol_t()
        s.n, s.cblknbr, s.bloknbr = self.n, self.cblknbr, self.bloknbr
        s.cb_fcol, s.cb_lcol, s.cb_fblok, s.bk_frow, s.bk_lrow, s.bk_fcblk = (a.ctypes.data_as(I64P) for a in self._arrs)
        self.s = s
        self.coefind = np.zeros(max(1, self.bloknbr), dtype=np.int64)
        self.coefnbr = int(load().ora_layout(C.byref(s), self.coefind.ctypes.data_as(I64P)))


def permuted_full(A: sps.spmatrix, perm: np.ndarray) -> sps.csc_matrix:
    """P A P^T with (P A P^T)[perm[i], perm[j]] = A[i, j], sorted CSC (int64)."""
    A = sps.coo_matrix(A)
    Ap = sps.coo_matrix((A.data, (perm[A.row], perm[A.col])), shape=A.shape).tocsc()
    Ap.sort_indices()
    return Ap


def factor(sym: Symbol, Ap: sps.csc_matrix, fact: str, crit: float, single: bool = False, nthreads: int = 1):
    """Fill and factorize; returns (L, U or None, static pivot count) in the 2D layout."""
    lib = load()
    dt = np.float32 if single else np.float64
    L = np.zeros(max(1, sym.coefnbr), dtype=dt)
    U = np.zeros_like(L) if fact == "GETRF" else None
    cp = np.ascontiguousarray(Ap.indptr, dtype=np.int64)
    ri = np.ascontiguousarray(Ap.indices, dtype=np.int64)
    va = np.ascontiguousarray(Ap.data, dtype=np.float64)
    fill = lib.ora_fill_s if single else lib.ora_fill_d
    rc = fill(C.byref(sym.s), sym.coefind.ctypes.data_as(I64P), FACT[fact], cp.ctypes.data_as(I64P),
              ri.ctypes.data_as(I64P), va.ctypes.data_as(C.c_void_p), L.ctypes.data_as(C.c_void_p),
              U.ctypes.data_as(C.c_void_p) if U is not None else None)
    if rc != 0:
        raise RuntimeError("entry outside the symbolic structure")
    npiv = lib.ora_factor(C.byref(sym.s), sym.coefind.ctypes.data_as(I64P), FACT[fact], int(single), float(crit),
                          L.ctypes.data_as(C.c_void_p), U.ctypes.data_as(C.c_void_p) if U is not None else None,
                          int(nthreads))
    return L, U, int(npiv)


def to_panels(sym: Symbol, X: np.ndarray) -> np.ndarray:
    """2D-layout coefficients -> the product's panel layout (same length)."""
    info = sym.info
    out = np.zeros_like(X)
    arr = [np.ascontiguousarray(info[k], dtype=np.int64) for k in ("cb_coef", "cb_stride", "bk_rowoff")]
    load().ora_to_panels(C.byref(sym.s), sym.coefind.ctypes.data_as(I64P), *(a.ctypes.data_as(I64P) for a in arr),
                         C.c_int(X.dtype == np.float32), X.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
    return out


def solve(sym: Symbol, fact: str, L: np.ndarray, U, B: np.ndarray, trans: bool = False) -> np.ndarray:
    """Solve with the oracle factors on permuted vectors (FP64 arithmetic)."""
    X = np.asfortranarray(np.array(B, dtype=np.float64, copy=True))
    if X.ndim == 1:
        X = X.reshape(-1, 1, order="F")
    Ld = np.ascontiguousarray(L, dtype=np.float64)
    Ud = np.ascontiguousarray(U, dtype=np.float64) if U is not None else None
    load().ora_solve(C.byref(sym.s), sym.coefind.ctypes.data_as(I64P), FACT[fact], Ld.ctypes.data_as(C.c_void_p),
                     Ud.ctypes.data_as(C.c_void_p) if Ud is not None else None, C.c_int(int(trans)),
                     C.c_int64(X.shape[1]), X.ctypes.data_as(C.c_void_p), C.c_int64(X.shape[0]))
    return X


def criterion(Ap: sps.spmatrix, magn_ctrl: float = 0.0) -> float:
    """Static-pivot threshold (sopalin/pastix_task_sopalin.c:464-495)."""
    nrm = float(np.sqrt((Ap.data.astype(np.float64) ** 2).sum()))
    if magn_ctrl < 0:
        return -magn_ctrl
    if magn_ctrl == 0:
        return np.ldexp(1.0, -53) * nrm
    return magn_ctrl * nrm


# ---------------- refinement drivers (numpy restatement) ----------------
def refine_gmres(A, b, x, precond, eps=1e-12, itermax=250, im=25):
    """refinement/z_refine_gmres.c:49-371 (right preconditioned GMRES(im))."""
    normb = np.linalg.norm(b) or 1.0
    normx = np.linalg.norm(x)
    iters = 0
    while True:
        r = b - A @ x if normx > 0 else b.copy()
        resid = np.linalg.norm(r)
        if resid / normb <= eps:
            break
        V = [r / resid]
        W = []
        H = np.zeros((im + 1, im))
        cs, sn = np.zeros(im), np.zeros(im)
        g = np.zeros(im + 1)
        g[0] = resid
        i = -1
        while True:
            i += 1
            w = precond(V[i].copy())
            W.append(w)
            v = A @ w
            for j in range(i + 1):
                H[j, i] = v @ V[j]
                v = v - H[j, i] * V[j]
            nrm = np.linalg.norm(v)
            H[i + 1, i] = nrm
            V.append(v / nrm if nrm > 1e-50 else v)
            for j in range(i):
                t = H[j, i]
                H[j, i] = cs[j] * t + sn[j] * H[j + 1, i]
                H[j + 1, i] = cs[j] * H[j + 1, i] - sn[j] * t
            t = np.hypot(H[i, i], H[i + 1, i])
            if abs(t) <= eps:
                t = eps
            cs[i], sn[i] = H[i, i] / t, H[i + 1, i] / t
            g[i + 1] = -sn[i] * g[i]
            g[i] = cs[i] * g[i]
            H[i, i] = cs[i] * H[i, i] + sn[i] * H[i + 1, i]
            iters += 1
            if i + 1 >= im or abs(g[i + 1]) / normb <= eps or iters >= itermax:
                break
        m = i + 1
        y = np.linalg.solve(np.triu(H[:m, :m]), g[:m])
        x = x + np.column_stack(W) @ y
        normx = 1.0
        if iters >= itermax:
            break
    return x, iters


def refine_cg(A, b, x, precond, eps=1e-12, itermax=250):
    """refinement/z_refine_grad.c:49-175 (preconditioned CG)."""
    normb = np.linalg.norm(b) or 1.0
    r = b - A @ x if np.linalg.norm(x) > 0 else b.copy()
    z = precond(r.copy())
    p = z.copy()
    it = 0
    res = np.linalg.norm(r) / normb
    while res > eps and it < itermax:
        it += 1
        q = A @ p
        beta = r @ z
        alpha = beta / (q @ p)
        x = x + alpha * p
        r = r - alpha * q
        z = precond(r.copy())
        beta = (r @ z) / beta
        p = z + beta * p
        res = np.linalg.norm(r) / normb
    return x, it
