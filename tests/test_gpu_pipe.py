"""The pipelined tile refill (term words and entry records staged in shared memory
two tiles ahead, A.x and V values one tile ahead): on plans of at most 512-term
tiles it must give the bits of the direct refill and of the oracle -- outputs of one
term, pairs (added atomically), lists of up to ~70 terms over 16 decades of
magnitude, unit products (no values), products read straight from L.x, refills with
new values, and enough tiles that the stages wrap many times."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _small_tiles(P):
    P.replan(tile_budget=512, tile_max_terms=512, refill_threads=128)
    return P.set_refill_pipe(True)


def _both(P, Lx, d, Ax):
    import torch
    out = []
    for on in (True, False):
        P.set_refill_pipe(on)
        cx = torch.full((max(1, P.nnz),), float("nan"), dtype=torch.float64, device="cuda")
        P.fill(Lx, d, Ax, cx)
        torch.cuda.synchronize()
        out.append(cx[:P.nnz].cpu().numpy())
    P.set_refill_pipe(True)
    return out


def _bits(a):
    return np.ascontiguousarray(a).view(np.int64)


@pytest.mark.parametrize("case", ["btda_random", "long_lists", "headline_like"])
def test_pipelined_refill_matches_direct_and_oracle(sdl, orc, case):
    from sparsediff_linalg_b200.device import btda_product
    rng = np.random.default_rng({"btda_random": 1, "long_lists": 2, "headline_like": 3}[case])
    if case == "btda_random":
        m, nA, nB = 20000, 3000, 2500
        A = wl.fixed_rowlen_csr(m, nA, 5, rng)
        B = wl.fixed_rowlen_csr(m, nB, 3, rng)
    elif case == "long_lists":
        # every A row hits all 4 columns: outputs collect 1..71 terms
        m, nA, nB = 60000, 4, 6000
        A = wl.fixed_rowlen_csr(m, nA, 4, rng)
        A = (A[0], A[1], A[2] * 10.0 ** rng.integers(-8, 9, len(A[2])), A[3], A[4])
        lens = rng.integers(1, 3, m)
        B = wl.variable_rowlen_csr(m, nB, lens, rng)
    else:
        m, nA, nB = 100000, 50000, 40000
        A = wl.fixed_rowlen_csr(m, nA, 8, rng)
        B = wl.fixed_rowlen_csr(m, nB, 8, rng)
    d = rng.uniform(0.1, 10, m)
    P, Tr = btda_product(_T(A[0]), _T(A[1]), A[4], _T(B[0]), _T(B[1]), B[4])
    assert _small_tiles(P), "the plan's tiles must fit the pipelined refill"
    for rnd in range(2):
        if rnd:
            A = (A[0], A[1], rng.standard_normal(len(A[1])), A[3], A[4])
            B = (B[0], B[1], rng.standard_normal(len(B[1])), B[3], B[4])
            d = rng.uniform(0.1, 10, m)
        pipe, direct = _both(P, _T(B[2]), _T(d), _T(A[2]))
        assert np.array_equal(_bits(pipe), _bits(direct)), f"round {rnd}: pipelined != direct"
        wp, wi, wx = orc.btda(A, B, d)
        assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
        assert np.array_equal(_bits(pipe), _bits(wx)), f"round {rnd}: pipelined != oracle"


def test_pipelined_refill_unit_and_direct_lx(sdl, orc):
    """C = A B with no values on L (every entry value 1.0, no V read) and with L.x
    read straight as the entry values (no d, L in value order)."""
    from sparsediff_linalg_b200.device import Product
    rng = np.random.default_rng(4)
    A = wl.fixed_rowlen_csr(30000, 20000, 6, rng)
    B = wl.fixed_rowlen_csr(20000, 15000, 4, rng)
    P = Product(_T(A[0]), _T(A[1]), _T(B[0]), _T(B[1]), B[4])
    assert _small_tiles(P)
    for Lx in (None, _T(A[2])):
        pipe, direct = _both(P, Lx, None, _T(B[2]))
        assert np.array_equal(_bits(pipe), _bits(direct))
        Ax = A[2] if Lx is not None else np.ones(len(A[1]))
        wp, wi, wx = orc.spgemm((A[0], A[1], Ax, A[3], A[4]), B)
        assert np.array_equal(_bits(pipe), _bits(wx))
