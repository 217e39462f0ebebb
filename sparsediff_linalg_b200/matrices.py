"""Python handles over the upstream polymorphic matrix API (matrix.h / matmul.h)
of the CUDA library. Host value buffers are the library-owned CSR arrays; writing
them goes through ``set_values``, which bumps ``values_version`` exactly as a C
caller does with ``matrix_values_changed``."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import CSR_p, check, lib, matrix_p

_SIGS = {
    "new_sparse_matrix": (matrix_p, [CSR_p]),
    "new_sparse_matrix_alloc": (matrix_p, [C.c_int, C.c_int, C.c_int]),
    "free_matrix": (None, [matrix_p]),
    "copy_sparsity_matrices_alloc": (matrix_p, [matrix_p]),
    "transpose_matrices_alloc": (matrix_p, [matrix_p]),
    "transpose_matrices_fill_values": (None, [matrix_p, matrix_p]),
    "BTA_matrices_alloc": (matrix_p, [matrix_p, matrix_p]),
    "BTA_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p]),
    "BTDA_matrices_fill_values": (None, [matrix_p, C.c_void_p, matrix_p, matrix_p]),
    "DA_matrices_fill_values": (None, [C.c_void_p, matrix_p, matrix_p]),
    "ATA_matrices_alloc": (matrix_p, [matrix_p]),
    "ATDA_matrices_fill_values": (None, [matrix_p, C.c_void_p, matrix_p]),
    "BA_matrices_alloc": (matrix_p, [matrix_p, matrix_p]),
    "BA_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p]),
    "new_permuted_dense": (matrix_p, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "new_permuted_dense_full": (matrix_p, [C.c_int, C.c_int, C.c_void_p]),
    "new_stacked_pd": (matrix_p, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
}
_bound = False


def mlib():
    global _bound
    L = lib()
    if not _bound:
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


_to_csr_t = C.CFUNCTYPE(CSR_p, matrix_p)
_gather_alloc_t = C.CFUNCTYPE(matrix_p, matrix_p, C.POINTER(C.c_int), C.c_int)
_fill_t = C.CFUNCTYPE(None, matrix_p, matrix_p)


class Matrix:
    """Owning handle of a library matrix (freed with free_matrix)."""

    def __init__(self, ptr):
        if not ptr:
            raise RuntimeError(lib().sdl_last_error().decode())
        self.ptr = ptr

    # ---- handle fields
    @property
    def m(self):
        return self.ptr.contents.m

    @property
    def n(self):
        return self.ptr.contents.n

    @property
    def nnz(self):
        return self.ptr.contents.nnz

    @property
    def kind(self):
        return self.ptr.contents.kind

    @property
    def version(self):
        return self.ptr.contents.values_version

    def values(self):
        """Live view of the host value buffer."""
        h = self.ptr.contents
        return np.ctypeslib.as_array(h.x, shape=(max(1, h.nnz),))[: h.nnz]

    def set_values(self, x):
        self.values()[...] = x
        self.ptr.contents.values_version += 1  # matrix_values_changed

    def csr(self):
        """(p, i, x) copies of the to_csr view."""
        c = _to_csr_t(self.ptr.contents.to_csr)(self.ptr).contents
        p = np.ctypeslib.as_array(c.p, shape=(c.m + 1,)).copy()
        i = np.ctypeslib.as_array(c.i, shape=(max(1, c.nnz),))[: c.nnz].copy()
        x = np.ctypeslib.as_array(c.x, shape=(max(1, c.nnz),))[: c.nnz].copy()
        return p, i, x

    def free(self):
        if self.ptr:
            mlib().free_matrix(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # ---- vtable
    def row_gather(self, mp):
        mp = np.ascontiguousarray(mp, np.int32)
        out = _gather_alloc_t(self.ptr.contents.row_gather_alloc)(
            self.ptr, mp.ctypes.data_as(C.POINTER(C.c_int)), len(mp))
        return Matrix(out)

    def row_gather_fill(self, out):
        _fill_t(self.ptr.contents.row_gather_fill_values)(self.ptr, out.ptr)

    def row_reduce(self, group, m_out):
        g = np.ascontiguousarray(group, np.int32)
        out = _gather_alloc_t(self.ptr.contents.row_reduce_alloc)(
            self.ptr, g.ctypes.data_as(C.POINTER(C.c_int)), m_out)
        return Matrix(out)

    def row_reduce_fill(self, out):
        _fill_t(self.ptr.contents.row_reduce_fill_values)(self.ptr, out.ptr)

    # ---- products (self is the output C where it says so)
    def BTA_alloc_with(self, B):
        """C = B^T self."""
        return Matrix(mlib().BTA_matrices_alloc(self.ptr, B.ptr))

    def BTDA_fill(self, A, d, B):
        """self = B^T diag(d) A."""
        dd = None if d is None else np.ascontiguousarray(d, np.float64)
        mlib().BTDA_matrices_fill_values(A.ptr, None if dd is None else dd.ctypes.data, B.ptr, self.ptr)


class SparseMatrix(Matrix):
    @classmethod
    def from_csr(cls, p, i, x, m, n):
        L = mlib()
        nnz = int(p[-1])
        csr = L.new_CSR_matrix(m, n, nnz)
        s = csr.contents
        np.ctypeslib.as_array(s.p, shape=(m + 1,))[:] = p
        if nnz:
            np.ctypeslib.as_array(s.i, shape=(nnz,))[:] = i
            np.ctypeslib.as_array(s.x, shape=(nnz,))[:] = x
        return cls(L.new_sparse_matrix(csr))


def BTA(A, B):
    return Matrix(mlib().BTA_matrices_alloc(A.ptr, B.ptr))


def BTDA_fill(A, d, B, Cm):
    Cm.BTDA_fill(A, d, B)


def BA(B, A):
    return Matrix(mlib().BA_matrices_alloc(B.ptr, A.ptr))


def BA_fill(B, A, Cm):
    mlib().BA_matrices_fill_values(B.ptr, A.ptr, Cm.ptr)


def ATA(A):
    return Matrix(mlib().ATA_matrices_alloc(A.ptr))


def ATDA_fill(A, d, Cm):
    dd = None if d is None else np.ascontiguousarray(d, np.float64)
    mlib().ATDA_matrices_fill_values(A.ptr, None if dd is None else dd.ctypes.data, Cm.ptr)


def DA_fill(d, A, Cm):
    dd = np.ascontiguousarray(d, np.float64)
    mlib().DA_matrices_fill_values(dd.ctypes.data, A.ptr, Cm.ptr)


def copy_sparsity(A):
    return Matrix(mlib().copy_sparsity_matrices_alloc(A.ptr))


def transpose(A):
    return Matrix(mlib().transpose_matrices_alloc(A.ptr))


def transpose_fill(A, AT):
    mlib().transpose_matrices_fill_values(A.ptr, AT.ptr)


def permuted_dense(m, n, row_perm, col_perm, X):
    rp = np.ascontiguousarray(row_perm, np.int32)
    cp = np.ascontiguousarray(col_perm, np.int32)
    X = np.ascontiguousarray(X, np.float64)
    return Matrix(mlib().new_permuted_dense(m, n, len(rp), len(cp), rp.ctypes.data, cp.ctypes.data,
                                            X.ctypes.data))


def stacked_pd(m, n, blocks):
    """Takes ownership of the block handles (they must not be freed afterwards)."""
    arr = (C.c_void_p * max(1, len(blocks)))(*[C.cast(b.ptr, C.c_void_p) for b in blocks])
    out = Matrix(mlib().new_stacked_pd(m, n, len(blocks), arr, None, None))
    for b in blocks:
        b.ptr = None
    return out
