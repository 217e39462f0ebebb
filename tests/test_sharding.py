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
