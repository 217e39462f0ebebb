"""The staged direct refill (each tile's term words and entry records bulk-copied
into shared memory by one thread while the tile before it runs, completing on an
mbarrier): on the 128-thread small-tile plan and on the
default 256-thread plan it must give the bits of the plain direct refill and of the
oracle -- outputs of one term, pairs (added atomically), lists of up to ~70 terms over
16 decades of magnitude, unit products, products read straight from L.x, refills with
new values -- and the staged and pipelined switches exclude each other."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _bits(a):
    return np.ascontiguousarray(a).view(np.int64)


def _both(P, Lx, d, Ax):
    """(staged, plain) values of one refill; leaves the staged refill selected."""
    import torch
    out = []
    for on in (True, False):
        P.set_refill_staged(on)
        cx = torch.full((max(1, P.nnz),), float("nan"), dtype=torch.float64, device="cuda")
        P.fill(Lx, d, Ax, cx)
        torch.cuda.synchronize()
        out.append(cx[:P.nnz].cpu().numpy())
    assert P.set_refill_staged(True)
    return out


def _operands(case, rng):
    if case == "btda_random":
        m, nA, nB = 20000, 3000, 2500
        A = wl.fixed_rowlen_csr(m, nA, 5, rng)
        B = wl.fixed_rowlen_csr(m, nB, 3, rng)
    elif case == "long_lists":
        m, nA, nB = 60000, 4, 6000          # every A row hits all 4 columns: lists of 1..71 terms
        A = wl.fixed_rowlen_csr(m, nA, 4, rng)
        A = (A[0], A[1], A[2] * 10.0 ** rng.integers(-8, 9, len(A[2])), A[3], A[4])
        B = wl.variable_rowlen_csr(m, nB, rng.integers(1, 3, m), rng)
    else:
        m, nA, nB = 100000, 50000, 40000    # the headline shape
        A = wl.fixed_rowlen_csr(m, nA, 8, rng)
        B = wl.fixed_rowlen_csr(m, nB, 8, rng)
    return m, A, B


@pytest.mark.parametrize("plan", ["small_tiles", "default"])
@pytest.mark.parametrize("case", ["btda_random", "long_lists", "headline_like"])
def test_staged_refill_matches_plain_and_oracle(sdl, orc, case, plan):
    from sparsediff_linalg_b200.device import btda_product
    rng = np.random.default_rng({"btda_random": 11, "long_lists": 12, "headline_like": 13}[case])
    m, A, B = _operands(case, rng)
    d = rng.uniform(0.1, 10, m)
    P, Tr = btda_product(_T(A[0]), _T(A[1]), A[4], _T(B[0]), _T(B[1]), B[4])
    if plan == "small_tiles":
        P.replan(tile_budget=512, tile_max_terms=512, refill_threads=128)
    if not P.set_refill_staged(True):
        assert plan == "default", "the small-tile plan's tiles always fit the staged refill"
        pytest.skip("this default plan's largest tile does not fit the staged refill's slots")
    for rnd in range(2):
        if rnd:
            A = (A[0], A[1], rng.standard_normal(len(A[1])), A[3], A[4])
            B = (B[0], B[1], rng.standard_normal(len(B[1])), B[3], B[4])
            d = rng.uniform(0.1, 10, m)
        staged, plain = _both(P, _T(B[2]), _T(d), _T(A[2]))
        assert np.array_equal(_bits(staged), _bits(plain)), f"round {rnd}: staged != plain"
        wp, wi, wx = orc.btda(A, B, d)
        assert np.array_equal(P.Cp.cpu().numpy(), wp) and np.array_equal(P.Ci.cpu().numpy(), wi)
        assert np.array_equal(_bits(staged), _bits(wx)), f"round {rnd}: staged != oracle"


def test_staged_refill_unit_and_direct_lx(sdl, orc):
    """C = A B with no values on L (every entry value 1.0, no V read) and with L.x
    read straight as the entry values (no d, L in value order)."""
    from sparsediff_linalg_b200.device import Product
    rng = np.random.default_rng(14)
    A = wl.fixed_rowlen_csr(30000, 20000, 6, rng)
    B = wl.fixed_rowlen_csr(20000, 15000, 4, rng)
    P = Product(_T(A[0]), _T(A[1]), _T(B[0]), _T(B[1]), B[4])
    P.replan(tile_budget=512, tile_max_terms=512, refill_threads=128)
    assert P.set_refill_staged(True)
    for Lx in (None, _T(A[2])):
        staged, plain = _both(P, Lx, None, _T(B[2]))
        assert np.array_equal(_bits(staged), _bits(plain))
        Ax = A[2] if Lx is not None else np.ones(len(A[1]))
        wp, wi, wx = orc.spgemm((A[0], A[1], Ax, A[3], A[4]), B)
        assert np.array_equal(_bits(staged), _bits(wx))


def test_staged_and_pipelined_switches_exclude_each_other(sdl):
    from sparsediff_linalg_b200.device import btda_product
    rng = np.random.default_rng(15)
    m, A, B = _operands("btda_random", rng)
    P, Tr = btda_product(_T(A[0]), _T(A[1]), A[4], _T(B[0]), _T(B[1]), B[4])
    P.replan(tile_budget=512, tile_max_terms=512, refill_threads=128)
    assert P.set_refill_staged(True) and P.refill_staged() and not P.refill_pipelined()
    assert P.set_refill_pipe(True) and P.refill_pipelined() and not P.refill_staged()
    assert P.set_refill_staged(True) and not P.refill_pipelined()
    assert P.tuning()["refill"] == "staged"
