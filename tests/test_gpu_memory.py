"""The device block cache: plans rebuilt from freed blocks (the cache) and from the
driver again after sdl_release_cached_memory give the same structure and bits, and a
product destroyed while the cache is full of its blocks leaves the next one intact."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _build_and_fill(A, B, d):
    import torch
    from sparsediff_linalg_b200.device import btda_product
    P, Tr = btda_product(_T(A[0]), _T(A[1]), A[4], _T(B[0]), _T(B[1]), B[4])
    cx = torch.full((max(1, P.nnz),), float("nan"), dtype=torch.float64, device="cuda")
    P.fill(_T(B[2]), _T(d), _T(A[2]), cx)
    torch.cuda.synchronize()
    return P.Cp.cpu().numpy(), P.Ci.cpu().numpy(), cx[:P.nnz].cpu().numpy().view(np.int64)


def test_rebuilt_plans_from_cached_blocks_match(sdl, orc):
    rng = np.random.default_rng(31)
    m = 60000
    A = wl.fixed_rowlen_csr(m, 20000, 6, rng)
    B = wl.fixed_rowlen_csr(m, 15000, 5, rng)
    d = rng.uniform(0.1, 10, m)
    first = _build_and_fill(A, B, d)          # blocks from the driver, freed into the cache
    again = _build_and_fill(A, B, d)          # the same sizes: taken from the cache
    sdl.sdl_release_cached_memory()
    fresh = _build_and_fill(A, B, d)          # from the driver again
    for got in (again, fresh):
        for a, b in zip(first, got):
            assert np.array_equal(a, b)
    wp, wi, wx = orc.btda(A, B, d)
    assert np.array_equal(first[0], wp) and np.array_equal(first[1], wi)
    assert np.array_equal(first[2], np.ascontiguousarray(wx).view(np.int64))
    # a different, smaller product next: blocks up to twice its sizes are reused
    A2 = wl.fixed_rowlen_csr(m, 20000, 4, rng)
    B2 = wl.fixed_rowlen_csr(m, 15000, 3, rng)
    got = _build_and_fill(A2, B2, d)
    wp, wi, wx = orc.btda(A2, B2, d)
    assert np.array_equal(got[0], wp) and np.array_equal(got[1], wi)
    assert np.array_equal(got[2], np.ascontiguousarray(wx).view(np.int64))
