"""GPU parity of the device-resident extension API (operands in HBM, torch tensors
for memory only) against the CPU oracle, bit for bit."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


def T(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


def test_btda_device_fused_csc(sdl, orc):
    """B's values are read through the CSC->CSR position map (no CSC refresh)."""
    import torch
    from sparsediff_linalg_b200.device import btda_product
    rng = np.random.default_rng(21)
    A = wl.fixed_rowlen_csr(5000, 3000, 8, rng)
    B = wl.fixed_rowlen_csr(5000, 2500, 8, rng)
    d = rng.uniform(0.1, 10, 5000)
    P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
    Cx = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    P.fill(T(B[2]), T(d), T(A[2]), Cx)
    torch.cuda.synchronize()
    wp, wi, wx = orc.btda(A, B, d)
    assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
    assert np.array_equal(bits(Cx.cpu().numpy()), bits(wx))


def test_btda_row_slices_equal_the_whole_product(sdl, orc):
    """A single product split by output rows (as ranks would hold it): the slices'
    structures and values, concatenated, are the whole product's, bit for bit."""
    import torch
    from sparsediff_linalg_b200.device import btda_product, btda_product_rows
    from sparsediff_linalg_b200.sharding import btda_row_weights, row_ranges
    rng = np.random.default_rng(22)
    A = wl.fixed_rowlen_csr(6000, 3000, 8, rng)
    lens = rng.integers(1, 20, 6000)
    B = wl.variable_rowlen_csr(6000, 2500, lens, rng)
    d = rng.uniform(0.1, 10, 6000)
    P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
    Cx = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    vals = (T(B[2]), T(d), T(A[2]))
    P.fill(*vals, Cx)
    ranges = row_ranges(btda_row_weights(A[0], B[0], B[1], B[4]), 3)
    cp, ci, cx = [np.zeros(1, np.int32)], [], []
    for r0, r1 in ranges:
        Q, _ = btda_product_rows(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4], r0, r1, transpose=Tr)
        Qx = torch.empty(max(1, Q.nnz), dtype=torch.float64, device="cuda")
        Q.fill(*vals, Qx)
        torch.cuda.synchronize()
        assert Q.m == r1 - r0
        cp.append(Q.Cp.cpu().numpy()[1:] + cp[-1][-1])
        ci.append(Q.Ci.cpu().numpy())
        cx.append(Qx[:Q.nnz].cpu().numpy())
    torch.cuda.synchronize()
    assert np.array_equal(np.concatenate(cp), P.Cp.cpu().numpy())
    assert np.array_equal(np.concatenate(ci), P.Ci.cpu().numpy())
    assert np.array_equal(bits(np.concatenate(cx)), bits(Cx.cpu().numpy()))


def test_spgemm_row_slices_equal_the_whole_product(sdl):
    """C = A B of skewed operands (rows beyond the tile budget included) split by
    output rows: the slices, concatenated, are the whole product bit for bit."""
    import torch
    from sparsediff_linalg_b200.device import Product, spgemm_product_rows
    from sparsediff_linalg_b200.sharding import row_ranges, spgemm_row_weights
    (Ap, Ai, Ax), (Bp, Bi, Bx), _ = wl.skewed_device(seed=31, m=8000, n=8000, target=160_000, cap=3000)
    P = Product(Ap, Ai, Bp, Bi, 8000)
    Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda")
    P.fill(Ax, None, Bx, Cx)
    ranges = row_ranges(spgemm_row_weights(Ap.cpu().numpy(), Ai.cpu().numpy(), Bp.cpu().numpy()), 3)
    cp, ci, cx = [np.zeros(1, np.int32)], [], []
    for r0, r1 in ranges:
        Q, (s0, s1) = spgemm_product_rows(Ap, Ai, Bp, Bi, 8000, r0, r1)
        Qx = torch.empty(max(1, Q.nnz), dtype=torch.float64, device="cuda")
        Q.fill(Ax[s0:s1], None, Bx, Qx)
        torch.cuda.synchronize()
        assert Q.m == r1 - r0
        cp.append(Q.Cp.cpu().numpy()[1:] + cp[-1][-1])
        ci.append(Q.Ci.cpu().numpy())
        cx.append(Qx[:Q.nnz].cpu().numpy())
    assert np.array_equal(np.concatenate(cp), P.Cp.cpu().numpy())
    assert np.array_equal(np.concatenate(ci), P.Ci.cpu().numpy())
    assert np.array_equal(bits(np.concatenate(cx)), bits(Cx[:P.nnz].cpu().numpy()))


def test_kron_blocks(sdl, orc):
    import torch
    from sparsediff_linalg_b200.device import Product
    rng = np.random.default_rng(5)
    blocks, nL, mL, n = 4, 50, 40, 60
    Lp, Li, Lx, _, _ = wl.small_random_csr(mL, nL, 0.1, rng)
    A = wl.small_random_csr(blocks * nL, n, 0.1, rng)
    d = rng.uniform(0.5, 2, blocks * nL)
    P = Product(T(Lp), T(Li), T(A[0]), T(A[1]), n, blocks=blocks)
    Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda")
    P.fill(T(Lx), T(d), T(A[2]), Cx)
    torch.cuda.synchronize()
    wp, wi, wx = orc.gustavson(Lp, Li, Lx, mL, blocks, d, A[0], A[1], A[2], A[3], A[4])
    assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
    assert np.array_equal(bits(Cx[:P.nnz].cpu().numpy()), bits(wx))


def test_unit_L_product_is_row_reduce(sdl, orc):
    """A unit-valued L (no Lx) is upstream's row_reduce: C[g] = sum of rows with group g."""
    import torch
    from sparsediff_linalg_b200.device import Product, Transpose
    rng = np.random.default_rng(8)
    m, n, m_out = 3000, 700, 300
    A = wl.small_random_csr(m, n, 0.01, rng)
    group = rng.integers(0, m_out, m).astype(np.int32)
    G = Transpose(T(np.arange(m + 1, dtype=np.int32)), T(group), m, m_out)
    P = Product(G.Tp, G.Ti, T(A[0]), T(A[1]), n)
    Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda")
    P.fill(None, None, T(A[2]), Cx)
    torch.cuda.synchronize()
    wp, wi, wx = orc.row_reduce(A[0], A[1], A[2], m, n, group, m_out)
    assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
    assert np.array_equal(bits(Cx[:P.nnz].cpu().numpy()), bits(wx))


@pytest.mark.slow
def test_btda_full_size_config(sdl, orc):
    """The 100000 x 50000 / 100000 x 40000, 8-per-row configuration at full size."""
    import torch
    from sparsediff_linalg_b200.device import btda_product
    A, B, d = wl.btda(seed=1)
    P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
    Cx = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    P.fill(T(B[2]), T(d), T(A[2]), Cx)
    torch.cuda.synchronize()
    wp, wi, wx = orc.btda(A, B, d)
    assert P.nnz == len(wi)
    assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
    assert np.array_equal(bits(Cx.cpu().numpy()), bits(wx))


def test_sharded_csr_to_csc_one_rank_nccl(sdl):
    """The column-partitioned conversion on one NCCL rank with the library's stable
    grouping (its all-to-all exchanges stay on the device): the same CSC as the
    one-GPU transpose, bit for bit, and the same values after a refill."""
    import socket
    import torch
    import torch.distributed as dist
    from sparsediff_linalg_b200.device import Transpose, group_by_key
    from sparsediff_linalg_b200.sharding import ShardedCsrToCsc
    rng = np.random.default_rng(44)
    m, n = 3000, 2200
    A = wl.variable_rowlen_csr(m, n, rng.integers(0, 12, m), rng)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        p, i, x = T(A[0]), T(A[1]), T(A[2])
        S = ShardedCsrToCsc(p, i, 0, m, n, group_by_key, dist)
        tx = S.fill(x)
        R = Transpose(p, i, m, n)
        rx = torch.empty(max(1, i.numel()), dtype=torch.float64, device="cuda")
        R.fill(x, rx)
        torch.cuda.synchronize()
        assert (S.c0, S.c1) == (0, n)
        assert np.array_equal(S.Tp.cpu().numpy(), R.Tp.cpu().numpy())
        assert np.array_equal(S.Ti.cpu().numpy(), R.Ti.cpu().numpy())
        assert np.array_equal(bits(tx.cpu().numpy()), bits(rx[:i.numel()].cpu().numpy()))
        x2 = x * -3.0
        tx2 = S.fill(x2)
        R.fill(x2, rx)
        torch.cuda.synchronize()
        assert np.array_equal(bits(tx2.cpu().numpy()), bits(rx[:i.numel()].cpu().numpy()))
    finally:
        dist.destroy_process_group()
