"""Host-side helpers for calling the upstream-compatible C API from Python.

``HostCSR`` / ``HostCSC`` / ``HostCOO`` wrap numpy arrays in the C structs without
copying (the arrays stay owned by Python, so these structs must never be passed
to a ``free_*`` function). ``csr_from_ptr`` copies a library-owned ``CSR_matrix*``
back into numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import COO_matrix, CSC_matrix, CSR_matrix


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class _Host:
    _struct_t = CSR_matrix

    def __init__(self, p, i, x, m, n):
        # private copies: set_values must never write into the caller's arrays
        self.p = np.array(p, dtype=np.int32, copy=True)
        self.i = np.array(i, dtype=np.int32, copy=True)
        self.x = np.array(x, dtype=np.float64, copy=True)
        # keep 1-element buffers alive for empty matrices so pointers are valid
        if self.i.size == 0:
            self.i = np.zeros(1, np.int32)[:0]
        if self.x.size == 0:
            self.x = np.zeros(1, np.float64)[:0]
        self.m, self.n = int(m), int(n)
        self.nnz = int(self.p[-1]) if self.p.size else 0
        self.struct = self._struct_t(_p(self.p, C.c_int), _p(self.i, C.c_int),
                                     _p(self.x, C.c_double), self.m, self.n, self.nnz)

    @property
    def ref(self):
        return C.pointer(self.struct)

    def set_values(self, x):
        self.x[...] = x


class HostCSR(_Host):
    _struct_t = CSR_matrix


class HostCSC(_Host):
    _struct_t = CSC_matrix


class HostCOO:
    def __init__(self, rows, cols, x, m, n):
        self.rows = np.array(rows, np.int32, copy=True)
        self.cols = np.array(cols, np.int32, copy=True)
        self.x = np.array(x, np.float64, copy=True)
        self.m, self.n, self.nnz = int(m), int(n), len(self.rows)
        self.struct = COO_matrix(_p(self.rows, C.c_int), _p(self.cols, C.c_int),
                                 _p(self.x, C.c_double), None, self.m, self.n, self.nnz)

    @property
    def ref(self):
        return C.pointer(self.struct)


def csr_from_ptr(ptr, rows_attr: str = "m"):
    """Copies (p, i, x, m, n) out of a library-owned CSR_matrix* / CSC_matrix*.
    For a CSC pass rows_attr='n' (its offsets span the columns)."""
    s = ptr.contents
    nrows = getattr(s, rows_attr)
    p = np.ctypeslib.as_array(s.p, shape=(nrows + 1,)).copy()
    nnz = int(s.nnz)
    if nnz:
        i = np.ctypeslib.as_array(s.i, shape=(nnz,)).copy()
        x = np.ctypeslib.as_array(s.x, shape=(nnz,)).copy()
    else:
        i = np.zeros(0, np.int32)
        x = np.zeros(0, np.float64)
    return p, i, x, int(s.m), int(s.n)


def values_view(ptr):
    """Live numpy view of a library-owned CSR/CSC's value array."""
    s = ptr.contents
    return np.ctypeslib.as_array(s.x, shape=(max(1, int(s.nnz)),))[: int(s.nnz)]
