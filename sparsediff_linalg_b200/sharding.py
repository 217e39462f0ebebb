"""Sharding of independent products across ranks (one process per GPU).

Products of a batch share nothing, so a multi-GPU run partitions them and needs no
collective on the data path: every rank builds and refills its own share. The
partition balances the products' term counts (the refill cost) with the greedy
longest-processing-time rule, deterministically, so every rank computes the same
partition without communicating.
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
