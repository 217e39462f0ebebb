"""Batched refill engine: grouped persistent launches (graph-replayed) over many
products give exactly the bits of each product's own refill, and of the oracle,
with one group, the default groups and a group per few products (the entry
values of the next group computed on the side stream while a group refills)."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group_bytes", [None, 0, 1 << 19])
def test_batch_matches_per_product_fills(sdl, orc, group_bytes):
    import torch
    from sparsediff_linalg_b200.device import Batch, btda_product
    inst = wl.batched_device(seed=11, count=24, lo=200, hi=6000)
    prods, outs, refs, vals = [], [], [], []
    for k in inst:
        P, T = btda_product(k["Ap"], k["Ai"], k["n"], k["Bp"], k["Bi"], k["n"])
        prods.append((P, T))
        outs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda"))
        refs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda"))
    B = Batch([p for p, _ in prods])
    if group_bytes is not None:
        B.set_group_bytes(group_bytes)
    if group_bytes == 0:
        assert B.groups == 1
    if group_bytes == 1 << 19:
        assert B.groups >= 5
    s = torch.cuda.Stream()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    for rnd in range(3):  # the first refill runs eagerly, the next ones replay the graph
        vals = []
        for i, k in enumerate(inst):
            ax = torch.randn(k["Ai"].numel(), generator=gen, device="cuda", dtype=torch.float64)
            bx = torch.randn(k["Bi"].numel(), generator=gen, device="cuda", dtype=torch.float64)
            d = torch.rand(k["m"], generator=gen, device="cuda", dtype=torch.float64) * 9.9 + 0.1
            vals.append((ax, bx, d))
            B.bind(i, bx, d, ax, outs[i])
        with torch.cuda.stream(s):
            B.refill(stream=s)
        s.synchronize()
        for i, (P, _) in enumerate(prods):
            ax, bx, d = vals[i]
            P.fill(bx, d, ax, refs[i])
        torch.cuda.synchronize()
        for i, (P, _) in enumerate(prods):
            got = outs[i][:P.nnz].cpu().numpy().view(np.int64)
            want = refs[i][:P.nnz].cpu().numpy().view(np.int64)
            assert np.array_equal(got, want), f"round {rnd}, product {i}"
    # one product against the oracle
    k = inst[3]
    ax, bx, d = [v.cpu().numpy() for v in vals[3]]
    A = (k["Ap"].cpu().numpy(), k["Ai"].cpu().numpy(), ax, k["m"], k["n"])
    Bm = (k["Bp"].cpu().numpy(), k["Bi"].cpu().numpy(), bx, k["m"], k["n"])
    wp, wi, wx = orc.btda(A, Bm, d)
    P = prods[3][0]
    assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
    assert np.array_equal(outs[3][:P.nnz].cpu().numpy().view(np.int64), wx.view(np.int64))
    # the unbatched path gives the same bits too
    with torch.cuda.stream(s):
        B.refill_unbatched(stream=s)
    s.synchronize()
    assert np.array_equal(outs[3][:P.nnz].cpu().numpy().view(np.int64), wx.view(np.int64))
    # the groups are fixed once the graph exists
    with pytest.raises(Exception):
        B.set_group_bytes(0)


def test_batch_with_heavy_rows_and_unit_products(sdl):
    """Products with rows beyond the tile budget (heavy-row term lists), a unit-valued
    product and small B^T D A products in one batch cut into several groups: every
    output is bit-identical to the product's own fill, eagerly and from the graph."""
    import torch
    from sparsediff_linalg_b200.device import Batch, Product, btda_product
    gen = torch.Generator(device="cuda")
    gen.manual_seed(9)
    prods, keep, vals = [], [], []
    for seed in (41, 42):
        (Ap, Ai, Ax), (Bp, Bi, Bx), _ = wl.skewed_device(seed=seed, m=6000, n=6000, target=120_000, cap=2000)
        keep.append((Ap, Ai, Bp, Bi))
        prods.append(Product(Ap, Ai, Bp, Bi, 6000))
        vals.append(lambda Ai=Ai, Bi=Bi: (torch.randn(Ai.numel(), generator=gen, device="cuda",
                                                      dtype=torch.float64), None,
                                          torch.randn(Bi.numel(), generator=gen, device="cuda",
                                                      dtype=torch.float64)))
    # the last structure again, unit-valued (no L values, no d)
    Ap, Ai, Bp, Bi = keep[-1]
    prods.append(Product(Ap, Ai, Bp, Bi, 6000))
    vals.append(lambda Bi=Bi: (None, None, torch.randn(Bi.numel(), generator=gen, device="cuda",
                                                       dtype=torch.float64)))
    for k in wl.batched_device(seed=12, count=6, lo=300, hi=3000):
        P, T = btda_product(k["Ap"], k["Ai"], k["n"], k["Bp"], k["Bi"], k["n"])
        keep.append(T)
        prods.append(P)
        vals.append(lambda k=k: (torch.randn(k["Bi"].numel(), generator=gen, device="cuda", dtype=torch.float64),
                                 torch.rand(k["m"], generator=gen, device="cuda", dtype=torch.float64) + 0.5,
                                 torch.randn(k["Ai"].numel(), generator=gen, device="cuda",
                                             dtype=torch.float64)))
    B = Batch(prods)
    assert B.big_rows > 0
    B.set_group_bytes(1 << 18)
    assert B.groups >= 3
    outs = [torch.full((max(1, P.nnz),), float("nan"), dtype=torch.float64, device="cuda") for P in prods]
    refs = [torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda") for P in prods]
    s = torch.cuda.Stream()
    for rnd in range(3):
        cur = [v() for v in vals]
        for i, (lx, d, ax) in enumerate(cur):
            B.bind(i, lx, d, ax, outs[i])
        with torch.cuda.stream(s):
            B.refill(stream=s)
        s.synchronize()
        for i, P in enumerate(prods):
            lx, d, ax = cur[i]
            P.fill(lx, d, ax, refs[i])
        torch.cuda.synchronize()
        for i, P in enumerate(prods):
            got = outs[i][:P.nnz].cpu().numpy().view(np.int64)
            want = refs[i][:P.nnz].cpu().numpy().view(np.int64)
            assert np.array_equal(got, want), f"round {rnd}, product {i}"


def test_batch_autotune_keeps_the_bits(sdl):
    """The batch autotuner times its candidate group sizes before the graph exists;
    the refill it settles on is bit-identical to each product's own fill."""
    import torch
    from sparsediff_linalg_b200.device import Batch, btda_product
    inst = wl.batched_device(seed=13, count=16, lo=500, hi=8000)
    prods, outs, refs = [], [], []
    for k in inst:
        P, T = btda_product(k["Ap"], k["Ai"], k["n"], k["Bp"], k["Bi"], k["n"])
        prods.append((P, T))
        outs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda"))
        refs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda"))
    B = Batch([p for p, _ in prods])
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    vals = []
    for i, k in enumerate(inst):
        v = (torch.randn(k["Ai"].numel(), generator=g, device="cuda", dtype=torch.float64),
             torch.randn(k["Bi"].numel(), generator=g, device="cuda", dtype=torch.float64),
             torch.rand(k["m"], generator=g, device="cuda", dtype=torch.float64) * 9.9 + 0.1)
        vals.append(v)
        B.bind(i, v[1], v[2], v[0], outs[i])
    s = torch.cuda.Stream()
    gb, ms = B.autotune(reps=2, stream=s)
    assert gb in (16 << 20, 32 << 20, 64 << 20, 128 << 20, 256 << 20, 0) and ms > 0
    with torch.cuda.stream(s):
        B.refill(stream=s)   # eager, then captured
        B.refill(stream=s)   # graph replay
    s.synchronize()
    for i, (P, _) in enumerate(prods):
        ax, bx, d = vals[i]
        P.fill(bx, d, ax, refs[i])
    torch.cuda.synchronize()
    for i, (P, _) in enumerate(prods):
        assert np.array_equal(outs[i][:P.nnz].cpu().numpy().view(np.int64),
                              refs[i][:P.nnz].cpu().numpy().view(np.int64)), i
    with pytest.raises(Exception):
        B.autotune(reps=1, stream=s)    # the graph exists: groups are fixed
