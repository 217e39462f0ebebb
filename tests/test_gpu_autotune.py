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
