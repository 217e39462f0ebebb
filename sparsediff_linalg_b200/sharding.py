"""Sharding across ranks (one process per GPU), with no collective on the data path.

* Independent products (a batch): products share nothing, so every rank builds and
  refills its own share. The partition balances the products' term counts (the
  refill cost) with the greedy longest-processing-time rule, deterministically, so
  every rank computes the same partition without communicating.
* One large product, by output rows: output row i of C = kron(I, L) diag(d) A
  depends on row i of L and on the rows of A it references only, so contiguous
  ranges of output rows are independent products over slices of L (A, d and the
  value arrays are read whole). `row_ranges` balances the ranges by the rows' term
  counts (`btda_row_weights` for C = B^T D A, `spgemm_row_weights` for C = A B);
  the outputs stay row-partitioned (rank r holds rows r0..r1 of C).
* CSR -> CSC of a row-partitioned matrix into a column-partitioned one
  (`ShardedCsrToCsc`): the one place with an exchange step. Column ranges are
  balanced by the columns' entry counts (one all-reduce of the counts per
  pattern); one all-to-all moves every entry to the rank of its column, and a value
  refill is one all-to-all of the values.
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


def spgemm_row_weights(A_p, A_i, B_p):
    """Terms of every output row of C = A B (host CSR structures): row i sums the
    lengths of the B rows that row i of A touches."""
    import numpy as np
    A_p = np.asarray(A_p, np.int64)
    lens_b = np.diff(np.asarray(B_p, np.int64))
    t = lens_b[np.asarray(A_i, np.int64)]
    pref = np.concatenate([[0], np.cumsum(t)])
    return pref[A_p[1:]] - pref[A_p[:-1]]


class ShardedCsrToCsc:
    """CSR -> CSC of an m x n matrix whose rows are spread over the ranks of a group
    (rank r holds rows r0 .. r0 + len(p) - 2: contiguous ranges, in rank order) into
    a CSC spread by columns (rank r gets columns c0 .. c1 - 1, ranges balanced by the
    columns' entry counts). Within every column the rows come out ascending, ties
    in row-major order: the one-GPU conversion's (and upstream's) order.

    The plan (once per pattern) exchanges the entries' rows and columns with one
    all-to-all; `fill(x)` exchanges the values with one more and returns this rank's
    CSC values. p, i (int32) and x (float64) are this rank's CSR rows (p relative,
    p[0] == 0). `group_by(keys, nkeys)` is a stable grouping of positions by key
    returning an object with `offsets` (nkeys + 1), `perm` (positions in key order,
    ties in position order) and `gather(x)` (x[perm]); on the GPU it is
    `device.group_by_key` (the library's stable transpose). `dist` is
    torch.distributed (NCCL for device tensors)."""

    def __init__(self, p, i, r0, m, n, group_by, dist, group=None):
        import torch
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        dev = i.device
        self.dist, self.group, self.n = dist, group, n
        nnz = int(i.numel())
        ranks_rows = [None] * world
        dist.all_gather_object(ranks_rows, (int(r0), int(p.numel()) - 1), group=group)
        start = 0
        for a, rows in ranks_rows:
            if a != start:
                raise ValueError("the ranks' row ranges must be contiguous and in rank order")
            start += rows
        if start != m:
            raise ValueError("the ranks' row ranges must cover the m rows")
        counts = torch.bincount(i.long(), minlength=n) if nnz else torch.zeros(n, dtype=torch.int64, device=dev)
        dist.all_reduce(counts, group=group)
        ranges = row_ranges(counts.cpu().numpy(), world)
        self.c0, self.c1 = ranges[rank]
        bounds = torch.tensor([a for a, _ in ranges[1:]], dtype=torch.int64, device=dev)
        dest = torch.searchsorted(bounds, i.long(), right=True).to(torch.int32)
        self._send = group_by(dest, world)
        send_counts = (self._send.offsets[1:] - self._send.offsets[:-1]).to(torch.int64)
        recv_counts = torch.empty_like(send_counts)
        dist.all_to_all_single(recv_counts, send_counts, group=group)
        self._sc = send_counts.cpu().tolist()
        self._rc = recv_counts.cpu().tolist()
        lens = (p[1:] - p[:-1]).long()
        rows = (torch.repeat_interleave(torch.arange(int(p.numel()) - 1, device=dev), lens) + r0).to(torch.int32)
        perm = self._send.perm.long()
        rrows = self._exchange(rows[perm], torch.int32)
        rcols = self._exchange(i[perm], torch.int32)
        self._recv = group_by((rcols - self.c0).to(torch.int32), self.c1 - self.c0)
        self.Tp = self._recv.offsets
        self.Ti = rrows[self._recv.perm.long()]
        self.nnz = int(rrows.numel())

    def _exchange(self, send, dtype):
        import torch
        recv = torch.empty(sum(self._rc), dtype=dtype, device=send.device)
        self.dist.all_to_all_single(recv, send.contiguous(), self._rc, self._sc, group=self.group)
        return recv

    def fill(self, x):
        """This rank's CSC values for new CSR values x (one all-to-all)."""
        import torch
        return self._recv.gather(self._exchange(self._send.gather(x), torch.float64))
