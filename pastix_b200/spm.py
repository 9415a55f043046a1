"""Minimal SpM matrix descriptor for the Python interface.

PaStiX takes its input as an ``spmatrix_t`` from the SpM library (not part of
the reference checkout).  :class:`spmatrix` builds that descriptor from a
SciPy sparse matrix, keeping the CSC arrays alive: ``SpmGeneral`` stores the
whole matrix, ``SpmSymmetric`` stores the lower triangle only.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np
import scipy.sparse as sps

from ._lib import PINT, spmatrix_t


class mtxtype(IntEnum):
    General = 111
    Symmetric = 112
    Hermitian = 113
    SymPosDef = 112  # positive definiteness is not a storage property
    HerPosDef = 113


class coeftype(IntEnum):
    Pattern = 0
    Float = 2
    Double = 3
    Complex32 = 4
    Complex64 = 5


class spmatrix:
    """CSC descriptor of a real matrix (int64 indices, float64 values)."""

    def __init__(self, A, mtxtype_: int | None = None, baseval: int = 0):
        A = sps.csc_matrix(A)
        A.sort_indices()
        A.sum_duplicates()
        if A.shape[0] != A.shape[1]:
            raise ValueError("square matrix expected")
        if mtxtype_ is None:
            mtxtype_ = mtxtype.General
        self.mtxtype = int(mtxtype_)
        if self.mtxtype == mtxtype.Symmetric:
            A = sps.tril(A, format="csc")
            A.sort_indices()
        self.A = A
        self.n = A.shape[0]
        self.colptr = np.ascontiguousarray(A.indptr.astype(np.int64) + baseval)
        self.rowptr = np.ascontiguousarray(A.indices.astype(np.int64) + baseval)
        self.values = np.ascontiguousarray(A.data.astype(np.float64))
        self.nnz = int(self.values.size)
        s = spmatrix_t()
        s.mtxtype = self.mtxtype
        s.flttype = int(coeftype.Double)
        s.fmttype = 0
        s.baseval = baseval
        s.gN = s.n = self.n
        s.gnnz = s.nnz = self.nnz
        s.gNexp = s.nexp = self.n
        s.gnnzexp = s.nnzexp = self.nnz
        s.dof = 1
        s.colptr = self.colptr.ctypes.data_as(PINT)
        s.rowptr = self.rowptr.ctypes.data_as(PINT)
        s.values = self.values.ctypes.data_as(C.c_void_p)
        self.spm = s

    def set_values(self, values: np.ndarray) -> None:
        """Replace the values (same pattern, same order as ``self.values``)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape != self.values.shape:
            raise ValueError("values shape mismatch")
        self.values[...] = v

    def full(self) -> sps.csc_matrix:
        """The full matrix (symmetric storage expanded)."""
        if self.mtxtype == mtxtype.Symmetric:
            L = self.A
            return (L + sps.tril(L, -1).T).tocsc()
        return self.A

    def pointer(self):
        return C.byref(self.spm)
