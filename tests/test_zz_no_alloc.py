"""sdl_product_fill_noalloc: the refill for callers that cannot call cudaMalloc
while they refill (device memory wholly owned by another allocator, a fixed
device-memory budget, or a latency-critical loop that must not pay cudaMalloc's
implicit synchronisation). It keeps the scratch of the rows with more than 8192
outputs in a fixed array inside the library instead of memory allocated for the
product, and must give exactly the bits of sdl_product_fill.

This file is collected last on purpose: if it fails, a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _operands(rng, nA=30000):
    """B^T D A whose output rows span the tile rows, the shared-accumulator rows and
    rows with more than 8192 outputs (the ones that use the scratch)."""
    m = 6000
    col_lens = [0, 1, 3, 8, 30, 100, 400, 1500, 3000, 6000] + [4] * 100
    ent = []
    for c, ln in enumerate(col_lens):
        rows = rng.choice(m, size=min(ln, m), replace=False)
        ent.append(np.stack([rows, np.full(len(rows), c)], 1))
    ent = np.concatenate(ent)
    ent = ent[np.lexsort((ent[:, 1], ent[:, 0]))]
    Bp = np.zeros(m + 1, np.int32)
    np.add.at(Bp, ent[:, 0] + 1, 1)
    Bp = np.cumsum(Bp).astype(np.int32)
    B = (Bp, ent[:, 1].astype(np.int32), rng.standard_normal(len(ent)), m, len(col_lens))
    A = wl.fixed_rowlen_csr(m, nA, 20, rng)
    return A, B


def test_noalloc_refill_matches_regular_fill(sdl):
    import torch
    from sparsediff_linalg_b200.device import btda_product

    rng = np.random.default_rng(2024)
    A, B = _operands(rng)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
    row_nnz = np.diff(P.Cp.cpu().numpy())
    assert row_nnz.max() > 8192, "the case must include rows that use the scratch"
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    want = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    got = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    allocs = sdl.sdl_device_alloc_count()
    for call in range(2):  # two calls in a row, with new values each time
        ax = T(rng.standard_normal(len(A[1])))
        bx = T(rng.standard_normal(len(B[1])))
        d = T(rng.uniform(0.1, 10.0, A[3]))
        got.fill_(float("nan"))
        P.fill(bx, d, ax, want)
        st = sdl.sdl_product_fill_noalloc(P.handle, C.c_void_p(bx.data_ptr()), C.c_void_p(d.data_ptr()),
                                          C.c_void_p(ax.data_ptr()), C.c_void_p(got.data_ptr()), stream)
        assert st == 0, sdl.sdl_last_error()
        torch.cuda.synchronize()
        w = want.cpu().numpy().view(np.int64)
        g = got.cpu().numpy().view(np.int64)
        assert np.array_equal(w, g), f"call {call}: values differ from sdl_product_fill"
    assert sdl.sdl_device_alloc_count() == allocs, "the refills must not allocate"


def test_noalloc_products_of_different_widths_alternate(sdl):
    """Two products whose A differ in width, refilled alternately through the shared
    scratch: each call finds its rows' map slices as it needs them, whatever the
    call before it left in the array."""
    import torch
    from sparsediff_linalg_b200.device import btda_product

    rng = np.random.default_rng(2025)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    cases = []
    for nA in (30000, 12000):
        A, B = _operands(rng, nA)
        P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
        assert np.diff(P.Cp.cpu().numpy()).max() > 8192
        cases.append((A, B, P, Tr))
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    for call in range(4):
        A, B, P, _ = cases[call % 2]
        ax = T(rng.standard_normal(len(A[1])))
        bx = T(rng.standard_normal(len(B[1])))
        d = T(rng.uniform(0.1, 10.0, A[3]))
        want = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
        got = torch.full((P.nnz,), float("nan"), dtype=torch.float64, device="cuda")
        P.fill(bx, d, ax, want)
        st = sdl.sdl_product_fill_noalloc(P.handle, C.c_void_p(bx.data_ptr()), C.c_void_p(d.data_ptr()),
                                          C.c_void_p(ax.data_ptr()), C.c_void_p(got.data_ptr()), stream)
        assert st == 0, sdl.sdl_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(want.cpu().numpy().view(np.int64), got.cpu().numpy().view(np.int64)), f"call {call}"


def test_noalloc_rejects_products_beyond_the_scratch(sdl):
    """A with more columns than the scratch map holds is refused with a clear error."""
    import torch
    from sparsediff_linalg_b200.device import Product

    n = 4 * 1024 * 1024 + 1
    Ap = torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda")
    Ai = torch.tensor([0, n - 1], dtype=torch.int32, device="cuda")
    Lp = torch.tensor([0, 2], dtype=torch.int32, device="cuda")
    Li = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
    P = Product(Lp, Li, Ap, Ai, n)
    x = torch.ones(2, dtype=torch.float64, device="cuda")
    out = torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda")
    st = sdl.sdl_product_fill_noalloc(P.handle, C.c_void_p(x.data_ptr()), None, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(out.data_ptr()), None)
    assert st == 3  # SDL_ERR_INVALID
    assert b"at most 4194304 columns" in sdl.sdl_last_error()
