"""Checker side of the tests and of bench.py's CPU baseline (test infrastructure).

Two CPU implementations live here, both built by ``oracle/Makefile`` into
``oracle/_ref/``:

* ``port``: ``libsdl_oracle.so``, this repository's plain-C restatement of the
  upstream algorithms (``sdl_oracle.c``; every function cites the upstream lines
  it follows);
* ``reference``: ``libsdl_ref.so``, the upstream library itself compiled from its
  own C sources, called through its public API.

Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
PORT_LIB = REF_DIR / "libsdl_oracle.so"
REF_LIB = REF_DIR / "libsdl_ref.so"

ip = C.POINTER(C.c_int)
dp = C.POINTER(C.c_double)


def build(quiet: bool = True) -> None:
    """Compile the port (always) and the upstream library (when its sources exist)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(r.stdout)


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


_PORT = None
_REF = None


def port():
    global _PORT
    if _PORT is None:
        if not PORT_LIB.exists():
            build()
        L = C.CDLL(str(PORT_LIB))
        L.orc_gustavson_count.restype = C.c_longlong
        L.orc_gustavson_count.argtypes = [ip, ip, C.c_int, C.c_int, ip, ip, C.c_int, C.c_int, ip, ip]
        L.orc_gustavson_structure.restype = None
        L.orc_gustavson_structure.argtypes = [ip, ip, C.c_int, C.c_int, ip, ip, C.c_int, C.c_int, ip, ip, ip]
        L.orc_gustavson_values.restype = None
        L.orc_gustavson_values.argtypes = [ip, ip, dp, C.c_int, C.c_int, dp, ip, ip, dp, C.c_int,
                                           C.c_int, ip, ip, dp, dp]
        L.orc_transpose.restype = None
        L.orc_transpose.argtypes = [ip, ip, dp, C.c_int, C.c_int, ip, ip, dp, ip]
        L.orc_coalesce_count.restype = C.c_longlong
        L.orc_coalesce_count.argtypes = [ip, ip, C.c_int, C.c_int, C.c_int, ip]
        L.orc_coalesce_fill.restype = None
        L.orc_coalesce_fill.argtypes = [ip, ip, dp, C.c_int, C.c_int, C.c_int, ip, ip, dp]
        L.orc_row_gather_count.restype = C.c_longlong
        L.orc_row_gather_count.argtypes = [ip, ip, C.c_int, ip]
        L.orc_row_gather_fill.restype = None
        L.orc_row_gather_fill.argtypes = [ip, ip, dp, ip, C.c_int, ip, ip, dp]
        L.orc_row_reduce_count.restype = C.c_longlong
        L.orc_row_reduce_count.argtypes = [ip, ip, C.c_int, C.c_int, ip, C.c_int, ip]
        L.orc_row_reduce_fill.restype = None
        L.orc_row_reduce_fill.argtypes = [ip, ip, dp, C.c_int, C.c_int, ip, C.c_int, ip, ip, dp]
        L.orc_dense_btdb.restype = None
        L.orc_dense_btdb.argtypes = [dp, dp, dp, C.c_int, C.c_int, C.c_int, dp]
        _PORT = L
    return _PORT


def reference_available() -> bool:
    return REF_LIB.exists()


def reference():
    """The upstream library (compiled from its sources), with the upstream
    signatures bound. Raises if it was not built."""
    global _REF
    if _REF is None:
        if not REF_LIB.exists():
            raise RuntimeError("upstream library not built (oracle/_ref/libsdl_ref.so)")
        from sparsediff_linalg_b200._lib import UPSTREAM_SIGNATURES, bind, CSR_p, CSC_p, matrix_p
        L = C.CDLL(str(REF_LIB))
        bind(L, UPSTREAM_SIGNATURES)
        vp = C.c_void_p
        extra = {
            "new_sparse_matrix": (matrix_p, [CSR_p]),
            "free_matrix": (None, [matrix_p]),
            "BTA_matrices_alloc": (matrix_p, [matrix_p, matrix_p]),
            "BTDA_matrices_fill_values": (None, [matrix_p, vp, matrix_p, matrix_p]),
            "BTA_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p]),
            "BA_matrices_alloc": (matrix_p, [matrix_p, matrix_p]),
            "BA_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p]),
            "ATA_matrices_alloc": (matrix_p, [matrix_p]),
            "ATDA_matrices_fill_values": (None, [matrix_p, vp, matrix_p]),
            "new_permuted_dense": (matrix_p, [C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
            "new_stacked_pd": (matrix_p, [C.c_int, C.c_int, C.c_int, vp, vp, vp]),
            "copy_sparsity_matrices_alloc": (matrix_p, [matrix_p]),
            "transpose_matrices_alloc": (matrix_p, [matrix_p]),
            "transpose_matrices_fill_values": (None, [matrix_p, matrix_p]),
            "DA_matrices_fill_values": (None, [vp, matrix_p, matrix_p]),
            # internal upstream entry points (src/internal/stacked_pd_linalg.h)
            "BA_spd_csr_alloc": (matrix_p, [matrix_p, CSR_p]),
            "BA_spd_csr_fill_values": (None, [matrix_p, CSR_p, matrix_p]),
        }
        bind(L, extra)
        _REF = L
    return _REF


# ----------------------------------------------------------------- numpy helpers
def gustavson(Lp, Li, Lx, L_m, blocks, d, Ap, Ai, Ax, A_m, A_n):
    """(Cp, Ci, Cx) of C = kron(I_blocks, L) diag(d) A by the port."""
    L = port()
    Lp = np.ascontiguousarray(Lp, np.int32); Li = np.ascontiguousarray(Li, np.int32)
    Ap = np.ascontiguousarray(Ap, np.int32); Ai = np.ascontiguousarray(Ai, np.int32)
    Cp = np.zeros(L_m * blocks + 1, np.int32)
    work = np.zeros(max(1, A_n), np.int32)
    nnz = L.orc_gustavson_count(_ptr(Lp, C.c_int), _ptr(Li, C.c_int), L_m, blocks,
                                _ptr(Ap, C.c_int), _ptr(Ai, C.c_int), A_m, A_n,
                                _ptr(Cp, C.c_int), _ptr(work, C.c_int))
    if nnz < 0:
        raise OverflowError("nnz(C) exceeds INT_MAX")
    Ci = np.zeros(max(1, nnz), np.int32)
    L.orc_gustavson_structure(_ptr(Lp, C.c_int), _ptr(Li, C.c_int), L_m, blocks,
                              _ptr(Ap, C.c_int), _ptr(Ai, C.c_int), A_m, A_n,
                              _ptr(Cp, C.c_int), _ptr(Ci, C.c_int), _ptr(work, C.c_int))
    Cx = np.zeros(max(1, nnz), np.float64)
    if Ax is not None:
        Lx = None if Lx is None else np.ascontiguousarray(Lx, np.float64)
        d = None if d is None else np.ascontiguousarray(d, np.float64)
        Ax = np.ascontiguousarray(Ax, np.float64)
        dwork = np.zeros(max(1, A_n), np.float64)
        L.orc_gustavson_values(_ptr(Lp, C.c_int), _ptr(Li, C.c_int), _ptr(Lx, C.c_double), L_m,
                               blocks, _ptr(d, C.c_double), _ptr(Ap, C.c_int), _ptr(Ai, C.c_int),
                               _ptr(Ax, C.c_double), A_m, A_n, _ptr(Cp, C.c_int),
                               _ptr(Ci, C.c_int), _ptr(Cx, C.c_double), _ptr(dwork, C.c_double))
    return Cp, Ci[:nnz], Cx[:nnz]


def transpose(p, idx, x, rows, cols):
    """(Tp, Ti, Tx) of the stable transpose by the port."""
    L = port()
    p = np.ascontiguousarray(p, np.int32); idx = np.ascontiguousarray(idx, np.int32)
    nnz = int(p[rows])
    Tp = np.zeros(cols + 1, np.int32)
    Ti = np.zeros(max(1, nnz), np.int32)
    Tx = np.zeros(max(1, nnz), np.float64)
    xx = None if x is None else np.ascontiguousarray(x, np.float64)
    work = np.zeros(max(1, cols), np.int32)
    L.orc_transpose(_ptr(p, C.c_int), _ptr(idx, C.c_int), _ptr(xx, C.c_double), rows, cols,
                    _ptr(Tp, C.c_int), _ptr(Ti, C.c_int), _ptr(Tx, C.c_double), _ptr(work, C.c_int))
    return Tp, Ti[:nnz], Tx[:nnz]


def coalesce(rows, cols, x, m, n):
    L = port()
    rows = np.ascontiguousarray(rows, np.int32); cols = np.ascontiguousarray(cols, np.int32)
    x = np.ascontiguousarray(x, np.float64)
    nnz = len(rows)
    Cp = np.zeros(m + 1, np.int32)
    out = L.orc_coalesce_count(_ptr(rows, C.c_int), _ptr(cols, C.c_int), nnz, m, n, _ptr(Cp, C.c_int))
    Ci = np.zeros(max(1, out), np.int32)
    Cx = np.zeros(max(1, out), np.float64)
    L.orc_coalesce_fill(_ptr(rows, C.c_int), _ptr(cols, C.c_int), _ptr(x, C.c_double), nnz, m, n,
                        _ptr(Cp, C.c_int), _ptr(Ci, C.c_int), _ptr(Cx, C.c_double))
    return Cp, Ci[:out], Cx[:out]


def row_gather(Ap, Ai, Ax, mp):
    L = port()
    Ap = np.ascontiguousarray(Ap, np.int32); Ai = np.ascontiguousarray(Ai, np.int32)
    Ax = np.ascontiguousarray(Ax, np.float64); mp = np.ascontiguousarray(mp, np.int32)
    m_out = len(mp)
    Cp = np.zeros(m_out + 1, np.int32)
    nnz = L.orc_row_gather_count(_ptr(Ap, C.c_int), _ptr(mp, C.c_int), m_out, _ptr(Cp, C.c_int))
    Ci = np.zeros(max(1, nnz), np.int32)
    Cx = np.zeros(max(1, nnz), np.float64)
    L.orc_row_gather_fill(_ptr(Ap, C.c_int), _ptr(Ai, C.c_int), _ptr(Ax, C.c_double),
                          _ptr(mp, C.c_int), m_out, _ptr(Cp, C.c_int), _ptr(Ci, C.c_int),
                          _ptr(Cx, C.c_double))
    return Cp, Ci[:nnz], Cx[:nnz]


def row_reduce(Ap, Ai, Ax, m, n, group, m_out):
    L = port()
    Ap = np.ascontiguousarray(Ap, np.int32); Ai = np.ascontiguousarray(Ai, np.int32)
    Ax = np.ascontiguousarray(Ax, np.float64); group = np.ascontiguousarray(group, np.int32)
    Cp = np.zeros(m_out + 1, np.int32)
    nnz = L.orc_row_reduce_count(_ptr(Ap, C.c_int), _ptr(Ai, C.c_int), m, n, _ptr(group, C.c_int),
                                 m_out, _ptr(Cp, C.c_int))
    Ci = np.zeros(max(1, nnz), np.int32)
    Cx = np.zeros(max(1, nnz), np.float64)
    L.orc_row_reduce_fill(_ptr(Ap, C.c_int), _ptr(Ai, C.c_int), _ptr(Ax, C.c_double), m, n,
                          _ptr(group, C.c_int), m_out, _ptr(Cp, C.c_int), _ptr(Ci, C.c_int),
                          _ptr(Cx, C.c_double))
    return Cp, Ci[:nnz], Cx[:nnz]


def btda(A, B_csr, d):
    """C = B^T diag(d) A with A, B given as CSR tuples (p, i, x, m, n): the port."""
    Ap, Ai, Ax, m, nA = A
    Bp, Bi, Bx, mB, nB = B_csr
    Tp, Ti, Tx = transpose(Bp, Bi, Bx, mB, nB)
    return gustavson(Tp, Ti, Tx, nB, 1, d, Ap, Ai, Ax, m, nA)


def spgemm(A, B):
    """C = A B (A, B CSR tuples) by the port (L = A's rows)."""
    Ap, Ai, Ax, mA, nA = A
    Bp, Bi, Bx, mB, nB = B
    return gustavson(Ap, Ai, Ax, mA, 1, None, Bp, Bi, Bx, mB, nB)


def blocks_csr(blocks, Sp, Si, Sx, S_n):
    """C_k = B_k S[col_perm_k, :] for dense blocks [(X_k (m0 x n0), col_perm_k)], as
    upstream's BA_pd_csr_alloc / BA_pd_csr_fill_values
    (src/permuted_dense/permuted_dense_linalg.c:313-430): output columns are the
    union of the patterns of S's rows col_perm_k, ascending; every output is summed
    over the compact CSC of S[col_perm_k, :] in its order (row r of the block
    ascending, then S's entry order), from +0.0, one rounding per product and per
    sum. The compact CSC is built once per distinct col_perm; the sums run one
    term depth at a time over all columns (a column has at most one term at each
    depth, so every cell still sees its terms in order). Returns
    [(col_perm_C, C_k)] per block (numpy, float64). Test infrastructure only."""
    Sp = np.asarray(Sp, np.int64)
    Si = np.asarray(Si, np.int64)
    Sx = np.asarray(Sx, np.float64)
    plans = {}

    def plan(cperm):
        key = np.asarray(cperm, np.int64).tobytes()
        if key in plans:
            return plans[key]
        cp = np.asarray(cperm, np.int64)
        lens = Sp[cp + 1] - Sp[cp] if len(cp) else np.zeros(0, np.int64)
        tot = int(lens.sum())
        r = np.repeat(np.arange(len(cp), dtype=np.int64), lens)
        first = np.repeat(Sp[cp] - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) if tot else r
        q = first + np.arange(tot, dtype=np.int64)        # S entries, rows r ascending
        c = Si[q]
        o = np.argsort(c, kind="stable")                  # compact CSC order
        r, q, c = r[o], q[o], c[o]
        cols, start = np.unique(c, return_index=True)
        loc = np.searchsorted(cols, c)
        depth = np.arange(tot, dtype=np.int64) - start[loc] if tot else np.zeros(0, np.int64)
        levels = []
        for t in range(int(depth.max()) + 1 if tot else 0):
            s = depth == t
            levels.append((loc[s], r[s], q[s]))
        plans[key] = (cols.astype(np.int32), levels)
        return plans[key]

    out = []
    for X, cperm in blocks:
        X = np.asarray(X, np.float64)
        cols, levels = plan(cperm)
        C = np.zeros((X.shape[0], len(cols)))
        for loc, r, q in levels:
            C[:, loc] = C[:, loc] + X[:, r] * Sx[q][None, :]
        out.append((cols, C))
    return out


def blocks_ata(blocks, d, n):
    """A^T diag(d) A of dense blocks [(X_k, row_perm_k, col_perm_k)], as upstream's
    ATA_spd_alloc / ATDA_spd_fill_values (src/stacked_pd/stacked_pd_linalg.c:197-237
    with the coalescing of src/stacked_pd/stacked_pd_coalesce.c:150-381): per block
    P_k = X_k^T diag(d[row_perm_k]) X_k; output blocks grouped by the set of blocks
    whose col_perm holds a row (in order of first appearance, rows ascending), columns
    the union of their col_perms; each cell the partials summed from 0 in block
    order. Returns [(rows, cols, C_o, Cabs_o)] where Cabs is the same sum of |terms|
    (the scale of the rounding bound). Test infrastructure only."""
    parts = []
    for X, rp, cp in blocks:
        X = np.asarray(X, np.float64)
        dp = np.ones(X.shape[0]) if d is None else np.asarray(d, np.float64)[np.asarray(rp)]
        W = X * dp[:, None]
        parts.append((np.asarray(cp), X.T @ W, np.abs(X).T @ np.abs(W)))
    sig_of, order = {}, []
    for r in range(n):
        sig = tuple(k for k, (cp, _, _) in enumerate(parts) if r in set(cp.tolist()))
        if not sig:
            continue
        if sig not in sig_of:
            sig_of[sig] = []
            order.append(sig)
        sig_of[sig].append(r)
    out = []
    for sig in order:
        rows = np.array(sig_of[sig], np.int32)
        cols = np.unique(np.concatenate([parts[k][0] for k in sig])).astype(np.int32)
        Cv = np.zeros((len(rows), len(cols)))
        Ca = np.zeros_like(Cv)
        for k in sig:
            cp, Pk, Ak = parts[k]
            pos = {c: j for j, c in enumerate(cp.tolist())}
            ri = [pos[r] for r in rows.tolist()]
            cj = [j for j, c in enumerate(cols.tolist()) if c in pos]
            ck = [pos[c] for c in cols.tolist() if c in pos]
            Cv[:, cj] = Cv[:, cj] + Pk[np.ix_(ri, ck)]
            Ca[:, cj] = Ca[:, cj] + Ak[np.ix_(ri, ck)]
        out.append((rows, cols, Cv, Ca))
    return out
