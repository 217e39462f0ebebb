"""Seeded synthetic inputs with the shapes, sizes and value distributions of the
sparse-product benchmark configurations (no public dataset is involved).

* spgemm_small   A, B 2000x2000 CSR, 5 distinct uniform columns per row, values
                 U[-1, 1], seed 0 (C = A B).
* btda           A 100000x50000, B 100000x40000, 8 distinct uniform columns per row,
                 values N(0, 1), d U[0.1, 10] (C = B^T D A, 40000x50000).
* batched        instances with rows log-uniform in [1k, 64k], cols = rows / 2,
                 4..16 nnz per row, fixed patterns; refills draw new N(0, 1) values
                 and d ~ U[0.1, 10].
* transpose_big  1M x 1M CSR, 10 distinct uniform columns per row.
* coalesce_big   50M COO triplets over 1M x 1M: 35M distinct pairs plus 15M
                 duplicates drawn from them, shuffled.
* skewed         1M x 1M CSR with Zipf(1.5) row lengths scaled to ~20M nnz
                 (capped at 50k per row).

Every generator returns CSR tuples (p, i, x, m, n) of numpy arrays.
"""
from __future__ import annotations

import numpy as np


def fixed_rowlen_csr(m, n, k, rng, dist="normal", lo=-1.0, hi=1.0):
    """m x n CSR with k distinct uniformly drawn columns per row (sorted)."""
    k = min(k, n)
    cols = np.sort(rng.integers(0, n, size=(m, k), dtype=np.int64), axis=1)
    while True:
        dup = np.any(cols[:, 1:] == cols[:, :-1], axis=1) if k > 1 else np.zeros(m, bool)
        nd = int(dup.sum())
        if nd == 0:
            break
        cols[dup] = np.sort(rng.integers(0, n, size=(nd, k), dtype=np.int64), axis=1)
    p = np.arange(0, m * k + 1, k, dtype=np.int32)
    i = cols.reshape(-1).astype(np.int32)
    x = _values(rng, m * k, dist, lo, hi)
    return p, i, x, m, n


def variable_rowlen_csr(m, n, lens, rng, dist="normal", lo=-1.0, hi=1.0):
    """m x n CSR with lens[r] distinct uniform columns in row r (sorted)."""
    lens = np.minimum(np.asarray(lens, np.int64), n)
    p = np.zeros(m + 1, np.int64)
    np.cumsum(lens, out=p[1:])
    nnz = int(p[-1])
    i = np.empty(nnz, np.int32)
    # rows grouped by length so each group is drawn as one (rows, k) block
    for k in np.unique(lens):
        if k == 0:
            continue
        rows = np.nonzero(lens == k)[0]
        if k > n // 4:  # dense-ish rows: permutation prefix
            for r in rows:
                i[p[r]:p[r + 1]] = np.sort(rng.permutation(n)[:k])
            continue
        block = fixed_rowlen_csr(len(rows), n, int(k), rng, dist="normal")[1].reshape(len(rows), k)
        idx = (p[rows][:, None] + np.arange(k)[None, :]).reshape(-1)
        i[idx] = block.reshape(-1)
    x = _values(rng, nnz, dist, lo, hi)
    return p.astype(np.int32), i, x, m, n


def _values(rng, count, dist, lo, hi):
    if dist == "normal":
        return rng.standard_normal(count)
    return rng.uniform(lo, hi, count)


def spgemm_small(seed=0):
    rng = np.random.default_rng(seed)
    A = fixed_rowlen_csr(2000, 2000, 5, rng, dist="uniform", lo=-1.0, hi=1.0)
    B = fixed_rowlen_csr(2000, 2000, 5, rng, dist="uniform", lo=-1.0, hi=1.0)
    return A, B


def btda(seed=1, m=100_000, nA=50_000, nB=40_000, k=8):
    rng = np.random.default_rng(seed)
    A = fixed_rowlen_csr(m, nA, k, rng)
    B = fixed_rowlen_csr(m, nB, k, rng)
    d = rng.uniform(0.1, 10.0, m)
    return A, B, d


def batched(seed=3, count=512, lo=1_000, hi=64_000):
    """List of (A, B, d) instances for C = B^T D A with uneven sizes."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    out = []
    for r in rows:
        r = int(r)
        c = max(1, r // 2)
        la = rng.integers(4, 17, r)
        lb = rng.integers(4, 17, r)
        A = variable_rowlen_csr(r, c, la, rng)
        B = variable_rowlen_csr(r, c, lb, rng)
        d = rng.uniform(0.1, 10.0, r)
        out.append((A, B, d))
    return out


def transpose_big(seed=4, m=1_000_000, n=1_000_000, k=10):
    rng = np.random.default_rng(seed)
    return fixed_rowlen_csr(m, n, k, rng)


def coalesce_big(seed=5, m=1_000_000, n=1_000_000, unique=35_000_000, dups=15_000_000):
    """(rows, cols, x, m, n) triplets: `unique` distinct pairs + `dups` repeats, shuffled."""
    rng = np.random.default_rng(seed)
    keys = np.unique(rng.integers(0, m * n, size=int(unique * 1.01), dtype=np.int64))
    while keys.size < unique:
        extra = rng.integers(0, m * n, size=unique - keys.size + 1000, dtype=np.int64)
        keys = np.unique(np.concatenate([keys, extra]))
    keys = rng.permutation(keys)[:unique]
    rep = keys[rng.integers(0, unique, size=dups)]
    allk = rng.permutation(np.concatenate([keys, rep]))
    rows = (allk // n).astype(np.int32)
    cols = (allk % n).astype(np.int32)
    x = rng.standard_normal(allk.size)
    return rows, cols, x, m, n


def zipf_lengths(m, alpha, target, cap, rng):
    """Row lengths min(cap, ceil(s * z)) with z ~ Zipf(alpha) and s found by bisection
    so that the total is ~target. Returns (lengths, s)."""
    z = rng.zipf(alpha, m).astype(np.float64)
    lo, hi = 1e-9, 1.0
    for _ in range(80):
        s = 0.5 * (lo + hi)
        tot = np.minimum(cap, np.ceil(s * z)).sum()
        if tot > target:
            hi = s
        else:
            lo = s
    s = lo
    return np.minimum(cap, np.ceil(s * z)).astype(np.int64), s


def skewed(seed=0, m=1_000_000, n=1_000_000, alpha=1.5, target=20_000_000, cap=50_000):
    rng = np.random.default_rng(seed)
    la, sa = zipf_lengths(m, alpha, target, cap, rng)
    lb, sb = zipf_lengths(m, alpha, target, cap, rng)
    A = variable_rowlen_csr(m, n, la, rng)
    B = variable_rowlen_csr(m, n, lb, rng)
    return A, B, (sa, sb)


def small_random_csr(m, n, density, rng, dist="normal"):
    """Bernoulli pattern (rows may be empty), for edge-case tests."""
    mask = rng.random((m, n)) < density
    p = np.zeros(m + 1, np.int32)
    p[1:] = np.cumsum(mask.sum(axis=1))
    i = np.nonzero(mask)[1].astype(np.int32)
    x = _values(rng, int(p[-1]), dist, -1.0, 1.0)
    return p, i, x, m, n


def batched_device(seed=3, count=512, lo=1_000, hi=64_000, device="cuda"):
    """The batched configuration generated on the GPU (torch, seeded): `count`
    instances with rows r ~ log-uniform[lo, hi], cols = r // 2, and for A and B of
    every instance 4..16 (uniform) distinct uniform columns per row (sorted), N(0,1)
    values; d ~ U[0.1, 10]. Returns a list of dicts of device tensors
    (Ap, Ai, Ax, Bp, Bi, Bx, d, m, n)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    gc = torch.Generator()
    gc.manual_seed(seed)
    rows = torch.exp(torch.empty(count, dtype=torch.float64).uniform_(
        float(np.log(lo)), float(np.log(hi)), generator=gc)).long().tolist()
    out = []

    def one(m, n):
        draws = 20
        cols = torch.floor(torch.rand((m, draws), generator=g, device=device, dtype=torch.float64) * n).long()
        cols, _ = torch.sort(cols, dim=1)
        uniq = torch.ones_like(cols, dtype=torch.bool)
        uniq[:, 1:] = cols[:, 1:] != cols[:, :-1]
        want = torch.randint(4, 17, (m, 1), generator=g, device=device)
        rank = torch.cumsum(uniq.int(), dim=1)
        keep = uniq & (rank <= want)
        lens = keep.sum(dim=1)
        p = torch.zeros(m + 1, dtype=torch.int32, device=device)
        p[1:] = torch.cumsum(lens, 0).int()
        i = cols[keep].int()
        x = torch.randn(i.numel(), generator=g, device=device, dtype=torch.float64)
        return p, i, x

    for r in rows:
        m, n = int(r), max(1, int(r) // 2)
        Ap, Ai, Ax = one(m, n)
        Bp, Bi, Bx = one(m, n)
        d = torch.rand(m, generator=g, device=device, dtype=torch.float64) * 9.9 + 0.1
        out.append(dict(Ap=Ap, Ai=Ai, Ax=Ax, Bp=Bp, Bi=Bi, Bx=Bx, d=d, m=m, n=n))
    return out


def skewed_device(seed=0, m=1_000_000, n=1_000_000, alpha=1.5, target=20_000_000, cap=50_000,
                  device="cuda"):
    """A, B (m x n) generated on the GPU with Zipf(alpha) row lengths
    min(cap, ceil(s * z)) (s found by bisection so the total is ~target) and
    distinct uniform columns per row (sorted), N(0, 1) values. Returns
    ((Ap, Ai, Ax), (Bp, Bi, Bx), scales) as device tensors. The Zipf draws use
    numpy (seeded); columns and values use a seeded torch generator."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)

    def one():
        lens, sc = zipf_lengths(m, alpha, target, cap, rng)
        lens_t = torch.as_tensor(lens, device=device)
        nnz = int(lens.sum())
        p = torch.zeros(m + 1, dtype=torch.int64, device=device)
        p[1:] = torch.cumsum(lens_t, 0)
        row = torch.repeat_interleave(torch.arange(m, device=device), lens_t)
        # draw, sort within rows, redraw duplicates until every row is distinct
        col = torch.randint(0, n, (nnz,), generator=g, device=device)
        for _ in range(64):
            key = row * n + col
            key, order = torch.sort(key)
            col = col[order]
            dup = torch.zeros(nnz, dtype=torch.bool, device=device)
            dup[1:] = key[1:] == key[:-1]
            nd = int(dup.sum())
            if nd == 0:
                break
            col[dup] = torch.randint(0, n, (nd,), generator=g, device=device)
        key = row * n + col
        key, _ = torch.sort(key)
        col = (key % n).int()
        x = torch.randn(nnz, generator=g, device=device, dtype=torch.float64)
        return (p.int(), col, x), sc

    A, sa = one()
    B, sb = one()
    return A, B, (sa, sb)


def coalesce_device(seed=5, m=1_000_000, n=1_000_000, unique=35_000_000, dups=15_000_000, device="cuda"):
    """The coalescing configuration generated on the GPU (torch, seeded): `unique`
    distinct (row, col) pairs drawn uniformly over m x n, plus `dups` repeats drawn
    uniformly from those pairs, shuffled; N(0, 1) values. Returns (rows, cols, x, m, n)
    with int32 / float64 device tensors."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    total = m * n
    keys = torch.unique(torch.randint(0, total, (int(unique * 1.01) + 16,), generator=g, device=device))
    while keys.numel() < unique:
        extra = torch.randint(0, total, (unique - keys.numel() + 1000,), generator=g, device=device)
        keys = torch.unique(torch.cat([keys, extra]))
    keys = keys[torch.randperm(keys.numel(), generator=g, device=device)[:unique]]
    rep = keys[torch.randint(0, unique, (dups,), generator=g, device=device)]
    allk = torch.cat([keys, rep])
    allk = allk[torch.randperm(allk.numel(), generator=g, device=device)]
    rows = (allk // n).to(torch.int32)
    cols = (allk % n).to(torch.int32)
    x = torch.randn(allk.numel(), generator=g, device=device, dtype=torch.float64)
    return rows, cols, x, m, n
