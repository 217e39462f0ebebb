"""Multi-threaded drivers of the CPU port for full-size checks (test infrastructure).

The port (``libsdl_oracle.so``) is single-threaded C; ctypes releases the GIL
while a foreign call runs, so independent pieces of one check run on all host
cores from a thread pool. Every split used here leaves each output bit-identical
to the one-call result, because the split follows the independence of the
upstream algorithms:

* rows of C = kron(I, L) diag(d) A depend only on their own row of L
  (upstream ``src/sparse/gustavson.c:26-143`` visits each output row on its own),
  so L is cut into contiguous row ranges and the pieces are concatenated;
* coalesced output rows depend only on the triplets of that row, in their input
  order (upstream ``src/sparse/sparse_matrix.c:136-240`` groups by output row with
  a stable counting sort), so the triplets are split by row range, keeping their
  order, and each range is coalesced on its own;
* independent products (a batch) are simply mapped over the pool.

Nothing in the product package imports this module; ``bench.py`` uses it only in
its CPU leg.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import oracle


def threads_default() -> int:
    return max(1, min(32, os.cpu_count() or 1))


def balanced_ranges(weights, parts):
    """Contiguous [r0, r1) ranges of len(weights) rows with about equal weight."""
    w = np.asarray(weights, np.float64)
    m = len(w)
    if m == 0:
        return [(0, 0)]
    parts = max(1, min(parts, m))
    c = np.cumsum(w)
    total = c[-1] if c[-1] > 0 else 1.0
    cuts = [0]
    for k in range(1, parts):
        cuts.append(int(np.searchsorted(c, total * k / parts, side="left")) + 1)
    cuts.append(m)
    cuts = sorted(set(min(max(x, 0), m) for x in cuts))
    return [(a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a] or [(0, m)]


def _concat_rows(pieces, m):
    """Concatenate row-range results [(r0, r1, Cp, Ci, Cx)] into one CSR."""
    pieces = sorted(pieces, key=lambda t: t[0])
    Cp = np.zeros(m + 1, np.int64)
    off = 0
    for r0, r1, p, _, _ in pieces:
        Cp[r0 + 1:r1 + 1] = np.asarray(p[1:], np.int64) + off
        off += int(p[-1])
    if off > 2**31 - 1:
        raise OverflowError("nnz(C) exceeds INT_MAX")
    Ci = np.concatenate([np.asarray(t[3], np.int32) for t in pieces]) if pieces else np.zeros(0, np.int32)
    Cx = np.concatenate([np.asarray(t[4], np.float64) for t in pieces]) if pieces else np.zeros(0)
    return Cp.astype(np.int32), Ci[:off], Cx[:off]


def gustavson_rows(Lp, Li, Lx, d, Ap, Ai, Ax, A_m, A_n, threads=None, weights=None):
    """(Cp, Ci, Cx) of C = L diag(d) A by the port, L cut into row ranges that run
    on a thread pool. weights (per L row) balances the ranges; by default the
    number of terms of every row."""
    Lp = np.asarray(Lp, np.int64)
    L_m = len(Lp) - 1
    th = threads or threads_default()
    if weights is None:
        alen = np.diff(np.asarray(Ap, np.int64))
        per_entry = alen[np.asarray(Li, np.int64)] if len(Li) else np.zeros(0, np.int64)
        cs = np.concatenate([[0], np.cumsum(per_entry)])
        weights = cs[Lp[1:]] - cs[Lp[:-1]] + 1
    ranges = balanced_ranges(weights, 4 * th)

    def one(rg):
        r0, r1 = rg
        a, b = int(Lp[r0]), int(Lp[r1])
        p = (Lp[r0:r1 + 1] - a).astype(np.int32)
        i = np.ascontiguousarray(Li[a:b], np.int32)
        x = None if Lx is None else np.ascontiguousarray(Lx[a:b], np.float64)
        Cp, Ci, Cx = oracle.gustavson(p, i, x, r1 - r0, 1, d, Ap, Ai, Ax, A_m, A_n)
        return r0, r1, Cp, Ci, Cx

    with ThreadPoolExecutor(th) as ex:
        pieces = list(ex.map(one, ranges))
    return _concat_rows(pieces, L_m)


def spgemm(A, B, threads=None):
    """C = A B (CSR tuples (p, i, x, m, n)) by the port, rows of A on a thread pool."""
    Ap, Ai, Ax, mA, nA = A
    Bp, Bi, Bx, mB, nB = B
    return gustavson_rows(Ap, Ai, Ax, None, Bp, Bi, Bx, mB, nB, threads=threads)


def btda(A, B_csr, d, threads=None):
    """C = B^T diag(d) A (CSR tuples) by the port: B's stable transpose, then the
    product with its rows (B's columns) on a thread pool."""
    Ap, Ai, Ax, m, nA = A
    Bp, Bi, Bx, mB, nB = B_csr
    Tp, Ti, Tx = oracle.transpose(Bp, Bi, Bx, mB, nB)
    return gustavson_rows(Tp, Ti, Tx, d, Ap, Ai, Ax, m, nA, threads=threads)


def coalesce(rows, cols, x, m, n, threads=None):
    """COO -> CSR with duplicates summed in input order (the port, equal to
    upstream's row_reduce of the one-triplet-per-row CSR), the output rows cut into
    ranges whose triplets (kept in input order) are coalesced on a thread pool."""
    th = threads or threads_default()
    rows = np.asarray(rows, np.int32)
    cols = np.asarray(cols, np.int32)
    x = np.asarray(x, np.float64)
    counts = np.bincount(rows, minlength=m)
    ranges = balanced_ranges(counts + 1, 2 * th)
    order = np.argsort(rows, kind="stable")        # by row, input order inside a row
    starts = np.concatenate([[0], np.cumsum(counts)])

    def one(rg):
        r0, r1 = rg
        sel = order[starts[r0]:starts[r1]]
        Cp, Ci, Cx = oracle.coalesce(rows[sel] - r0, cols[sel], x[sel], r1 - r0, n)
        return r0, r1, Cp, Ci, Cx

    with ThreadPoolExecutor(th) as ex:
        pieces = list(ex.map(one, ranges))
    return _concat_rows(pieces, m)


def map_threads(fn, items, threads=None):
    with ThreadPoolExecutor(threads or threads_default()) as ex:
        return list(ex.map(fn, items))


def compare_csr(got, want, tol=1e-12):
    """Structure and value agreement of two CSR results (p, i, x): structure_equal
    (row offsets and column indices identical), bit_identical (values compared as
    int64 bit patterns), max_rel_err (max |got - want| / |want| over entries with
    want != 0, and |got| where want == 0), within_tol."""
    gp, gi, gx = (np.asarray(a) for a in got[:3])
    wp, wi, wx = (np.asarray(a) for a in want[:3])
    struct = bool(np.array_equal(gp.astype(np.int64), wp.astype(np.int64)) and
                  np.array_equal(gi.astype(np.int64), wi.astype(np.int64)))
    res = {"structure_equal": struct, "nnz": int(len(wi))}
    if not struct or len(gx) != len(wx):
        res.update(bit_identical=False, max_rel_err=None, within_tol=False)
        return res
    gx = np.ascontiguousarray(gx, np.float64)
    wx = np.ascontiguousarray(wx, np.float64)
    bits = bool(np.array_equal(gx.view(np.int64), wx.view(np.int64)))
    if bits:
        rel = 0.0
    else:
        den = np.abs(wx)
        diff = np.abs(gx - wx)
        nz = den > 0
        r1 = float(np.max(diff[nz] / den[nz])) if nz.any() else 0.0
        r0 = float(np.max(diff[~nz])) if (~nz).any() else 0.0
        rel = max(r1, r0)
    res.update(bit_identical=bits, max_rel_err=rel, within_tol=bool(rel <= tol))
    return res
