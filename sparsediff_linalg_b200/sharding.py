"""Sharding across ranks (one process per GPU), with no collective on the data path.

* Independent products (a batch): products share nothing, so every rank builds and
  refills its own share. The partition balances the products' term counts (the
  refill cost) with the greedy longest-processing-time rule, deterministically, so
  every rank computes the same partition without communicating.
* One large product, by output rows: output row i of C = kron(I, L) diag(d) A
  depends on row i of L and on the rows of A it references only, so contiguous
  ranges of output rows are independent products over slices of L (A, d and the
  value arrays are read whole). `row_ranges` balances the ranges by the rows' term
  counts; the outputs stay row-partitioned (rank r holds rows r0..r1 of C).
"""
from __future__ import annotations


def shard_products(weights, world_size):
    """Partition product indices 0..len(weights)-1 into `world_size` lists with
    balanced total weight (LPT: heaviest first onto the lightest rank; ties broken
    by index, so the result is the same on every rank)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    loads = [0] * world_size
    shards = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (loads[q], q))
        shards[r].append(i)
        loads[r] += weights[i]
    return [sorted(s) for s in shards]


def my_shard(weights, rank, world_size):
    return shard_products(weights, world_size)[rank]


def row_ranges(row_weights, world_size):
    """Contiguous, balanced ranges of output rows: a list of (r0, r1) per rank,
    covering 0..len(row_weights) in order. Rank r's range ends at the first row
    whose weight prefix reaches (r + 1) / world_size of the total, so the result
    depends on the weights only and is the same on every rank."""
    import numpy as np
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    w = np.asarray(row_weights, dtype=np.float64)
    if np.any(w < 0):
        raise ValueError("row weights must be non-negative")
    n = len(w)
    pref = np.concatenate([[0.0], np.cumsum(w)])
    total = pref[-1]
    cuts = [0]
    for r in range(1, world_size):
        c = int(np.searchsorted(pref, total * r / world_size, side="left")) if total > 0 else (n * r) // world_size
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


def btda_row_weights(A_p, B_p, B_i, B_n):
    """Terms of every output row of C = B^T diag(d) A (host CSR structures of A and
    B, same row count): row i sums the lengths of the A rows that column i of B
    touches."""
    import numpy as np
    A_p = np.asarray(A_p, np.int64)
    B_p = np.asarray(B_p, np.int64)
    lens = np.diff(A_p)
    rows_of_b = np.repeat(np.arange(len(B_p) - 1), np.diff(B_p))
    return np.bincount(np.asarray(B_i, np.int64), weights=lens[rows_of_b], minlength=B_n)
