"""The autotuner (sdl_product_autotune) only moves the schedule: every candidate
plan it builds is checked to have the exact structure of the original (row
offsets and column indices compared on the device), and the tuned product's
refill is bit-identical to the as-given product's."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


@pytest.mark.parametrize("case", ["btda", "wide_rows"])
def test_autotune_keeps_structure_and_values(sdl, case):
    import torch
    from sparsediff_linalg_b200.device import Product, btda_product
    rng = np.random.default_rng(900 + (case == "wide_rows"))
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    if case == "btda":
        A = wl.fixed_rowlen_csr(20000, 9000, 8, rng)
        B = wl.fixed_rowlen_csr(20000, 7000, 6, rng)
        keep = []

        def make():
            P, Tr = btda_product(T(A[0]), T(A[1]), A[4], T(B[0]), T(B[1]), B[4])
            keep.append(Tr)  # the product's L arrays live in the transpose plan
            return P
        Lx, Ax, d = T(B[2]), T(A[2]), T(rng.uniform(0.1, 10, 20000))
    else:
        # C = L A with rows of 100 to 700 terms: the warp-kernel threshold matters
        lens = rng.integers(10, 70, 3000)
        Lm = wl.variable_rowlen_csr(3000, 4000, lens, rng)
        A = wl.fixed_rowlen_csr(4000, 50000, 10, rng)
        make = lambda: Product(T(Lm[0]), T(Lm[1]), T(A[0]), T(A[1]), A[4])  # noqa: E731
        Lx, Ax, d = T(Lm[2]), T(A[2]), None
    P0 = make()
    C0 = torch.full((P0.nnz,), float("nan"), dtype=torch.float64, device="cuda")
    P0.fill(Lx, d, Ax, C0)
    P1 = make()
    tune = P1.autotune(reps=2)
    assert tune["candidates"] >= 10
    assert tune["refill_us"] > 0 and tune["refill_us"] <= tune["default_refill_us"] + 1e-9
    assert tune["warp_max_terms"] in (128, 512) and tune["rows_per_cta_warp"] in (4, 8, 16)
    assert tune["refill_ctas_per_sm"] in (0, 3, 4)
    assert torch.equal(P1.Cp, P0.Cp) and torch.equal(P1.Ci, P0.Ci)
    C1 = torch.full((P1.nnz,), float("nan"), dtype=torch.float64, device="cuda")
    P1.fill(Lx, d, Ax, C1)
    torch.cuda.synchronize()
    assert np.array_equal(bits(C1.cpu().numpy()), bits(C0.cpu().numpy()))
    assert tune["refill_threads"] in (128, 256)


@pytest.mark.parametrize("shape", [(512, 512, 128), (512, 1024, 128), (700, 0, 256), (0, 300, 256)])
def test_replan_refill_shapes_keep_values(sdl, shape):
    """Explicit refill configurations (sdl_product_replan): the small-tile refill
    (128-thread CTAs; tile rows above 512 terms leave the tiles for the larger-row
    kernels), a 128-thread request whose windows do not fit (it runs the 256-thread
    refill), other budgets and largest tile rows: structure and values unchanged."""
    import torch
    from sparsediff_linalg_b200.device import Product
    budget, tmax, threads = shape
    rng = np.random.default_rng(950)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    # rows of 40 to 900 terms, so a 300- or 512-term largest tile row moves rows out
    lens = rng.integers(4, 90, 4000)
    Lm = wl.variable_rowlen_csr(4000, 3000, lens, rng)
    A = wl.fixed_rowlen_csr(3000, 20000, 10, rng)
    Lx, Ax = T(Lm[2]), T(A[2])
    P0 = Product(T(Lm[0]), T(Lm[1]), T(A[0]), T(A[1]), A[4])
    C0 = torch.full((P0.nnz,), float("nan"), dtype=torch.float64, device="cuda")
    P0.fill(Lx, None, Ax, C0)
    P1 = Product(T(Lm[0]), T(Lm[1]), T(A[0]), T(A[1]), A[4])
    P1.replan(tile_budget=budget, tile_max_terms=tmax, refill_threads=threads)
    got_threads, got_max = P1.refill_shape()
    assert got_max == (tmax if tmax else 1024)
    if threads == 128 and budget <= 512 and 0 < tmax <= 512:
        assert got_threads == 128      # tiles then hold fewer than 1024 terms: the windows fit
    elif threads == 256:
        assert got_threads == 256
    else:
        assert got_threads in (128, 256)  # 128 only where every window fits
    assert torch.equal(P1.Cp, P0.Cp) and torch.equal(P1.Ci, P0.Ci)
    for rnd in range(2):
        C1 = torch.full((P1.nnz,), float("nan"), dtype=torch.float64, device="cuda")
        P1.fill(Lx, None, Ax, C1)
        torch.cuda.synchronize()
        assert np.array_equal(bits(C1.cpu().numpy()), bits(C0.cpu().numpy())), rnd
    with pytest.raises(Exception):
        P1.replan(refill_threads=64)
