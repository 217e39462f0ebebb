"""Multi-rank host logic on CPU (gloo, 2 ranks): every rank derives the same
balanced partition of independent products without exchanging data, and the
shards are disjoint, complete and balanced."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, weights, out):
    import torch
    import torch.distributed as dist
    from sparsediff_linalg_b200.sharding import my_shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = my_shard(weights, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    load = torch.tensor([sum(weights[i] for i in mine)], dtype=torch.float64)
    loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(loads, load)
    out.put((rank, gathered, [float(x) for x in loads]))
    dist.destroy_process_group()


def test_two_rank_partition_gloo():
    import multiprocessing as mp
    import random
    rnd = random.Random(3)
    weights = [rnd.randint(1_000, 640_000) for _ in range(512)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, weights, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, g0, l0), (_, g1, l1) = res
    assert g0 == g1, "every rank must see the same partition"
    a, b = set(g0[0]), set(g0[1])
    assert not (a & b) and (a | b) == set(range(512))
    assert abs(l0[0] - l0[1]) <= max(weights), "partition must be balanced"


@pytest.mark.parametrize("world", [1, 3, 8])
def test_partition_properties(world):
    from sparsediff_linalg_b200.sharding import shard_products
    weights = [(i * 7919) % 1000 + 1 for i in range(100)]
    shards = shard_products(weights, world)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(100))
    loads = [sum(weights[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(weights)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_row_ranges_contiguous_and_balanced(world):
    import numpy as np
    from sparsediff_linalg_b200.sharding import row_ranges
    rng = np.random.default_rng(5)
    w = rng.integers(0, 300, 10000).astype(float)
    w[:50] = 5000                                    # a heavy head
    rr = row_ranges(w, world)
    assert rr[0][0] == 0 and rr[-1][1] == len(w)
    assert all(a[1] == b[0] for a, b in zip(rr, rr[1:]))
    loads = [w[a:b].sum() for a, b in rr]
    assert max(loads) - min(loads) <= 2 * w.max()
    assert row_ranges(w, world) == rr                # deterministic


def test_btda_row_weights_matches_terms():
    import numpy as np
    from sparsediff_linalg_b200 import workloads as wl
    from sparsediff_linalg_b200.sharding import btda_row_weights
    rng = np.random.default_rng(6)
    A = wl.small_random_csr(40, 30, 0.2, rng)
    B = wl.small_random_csr(40, 25, 0.2, rng)
    w = btda_row_weights(A[0], B[0], B[1], 25)
    lens = np.diff(A[0])
    want = np.zeros(25)
    for k in range(40):
        for q in range(B[0][k], B[0][k + 1]):
            want[B[1][q]] += lens[k]
    assert np.array_equal(w, want)


def test_spgemm_row_weights_matches_terms():
    import numpy as np
    from sparsediff_linalg_b200 import workloads as wl
    from sparsediff_linalg_b200.sharding import row_ranges, spgemm_row_weights
    rng = np.random.default_rng(7)
    A = wl.small_random_csr(50, 35, 0.2, rng)
    B = wl.small_random_csr(35, 45, 0.3, rng)
    w = spgemm_row_weights(A[0], A[1], B[0])
    lens_b = np.diff(B[0])
    want = [sum(lens_b[A[1][q]] for q in range(A[0][i], A[0][i + 1])) for i in range(50)]
    assert np.array_equal(w, want)
    ranges = row_ranges(w, 4)
    assert ranges[0][0] == 0 and ranges[-1][1] == 50
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))


class _StableGroup:
    """numpy stable grouping (the CPU stand-in for the library's transpose)."""

    def __init__(self, keys, nkeys):
        import numpy as np
        import torch
        k = keys.numpy().astype(np.int64)
        self.perm = torch.as_tensor(np.argsort(k, kind="stable").astype(np.int32))
        self.offsets = torch.as_tensor(
            np.concatenate([[0], np.cumsum(np.bincount(k, minlength=nkeys))]).astype(np.int32))

    def gather(self, x):
        return x[self.perm.long()]


def _csc_worker(rank, world, port, csr, n, out):
    import torch
    import torch.distributed as dist
    from sparsediff_linalg_b200.sharding import ShardedCsrToCsc, row_ranges
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p, i, x = csr
    m = len(p) - 1
    a, b = row_ranges([1.0] * m, world)[rank]
    pl = torch.as_tensor(p[a:b + 1] - p[a])
    il = torch.as_tensor(i[p[a]:p[b]])
    xl = torch.as_tensor(x[p[a]:p[b]])
    S = ShardedCsrToCsc(pl, il, a, m, n, _StableGroup, dist)
    tx = S.fill(xl)
    tx2 = S.fill(-2.0 * xl)
    out.put((rank, S.c0, S.c1, S.Tp.numpy(), S.Ti.numpy(), tx.numpy(), tx2.numpy()))
    dist.destroy_process_group()


@pytest.mark.parametrize("world,m,n", [(2, 70, 55), (3, 70, 55), (4, 3, 5)])
def test_sharded_csr_to_csc_gloo(world, m, n):
    """Rows spread over `world` gloo ranks -> columns spread over them, with one
    all-to-all: reassembled, the CSC is the stable transpose (rows ascending in every
    column), and a value refill moves the new values the same way."""
    import multiprocessing as mp
    import numpy as np
    rng = np.random.default_rng(40 + world)
    dense = (rng.random((m, n)) < (0.12 if m > 10 else 0.5)) * rng.standard_normal((m, n))
    if m > 10:
        dense[5] = 0.0      # an empty row
        dense[:, 7] = 0.0   # an empty column
    # (4 ranks over 3 rows and 5 columns: one rank holds no rows, some hold no columns)
    p = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.int32)
    i = np.nonzero(dense)[1].astype(np.int32)
    x = dense[dense != 0].astype(np.float64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_csc_worker, args=(r, world, port, (p, i, x), n, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted([q.get(timeout=120) for _ in range(world)], key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert res[0][1] == 0 and res[-1][2] == n
    assert all(res[r][2] == res[r + 1][1] for r in range(world - 1))
    Tp = [np.zeros(1, np.int64)]
    Ti, Tx, Tx2 = [], [], []
    off = 0
    for _, c0, c1, tp, ti, tx, tx2 in res:
        assert len(tp) == c1 - c0 + 1 and tp[0] == 0 and tp[-1] == len(ti)
        Tp.append(tp[1:].astype(np.int64) + off)
        off += len(ti)
        Ti.append(ti)
        Tx.append(tx)
        Tx2.append(tx2)
    rows = np.repeat(np.arange(m), np.diff(p))
    order = np.argsort(i, kind="stable")
    want_p = np.concatenate([[0], np.cumsum(np.bincount(i, minlength=n))])
    assert np.array_equal(np.concatenate(Tp), want_p)
    assert np.array_equal(np.concatenate(Ti), rows[order])
    assert np.array_equal(np.concatenate(Tx), x[order])
    assert np.array_equal(np.concatenate(Tx2), -2.0 * x[order])
