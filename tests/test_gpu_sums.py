"""Matrix sums and vstack through the drop-in C ABI against the same calls on the
upstream library compiled from its sources (upstream src/sparse/matrix_sum.c,
src/sparse/CSR_sum.c, src/sparse/matrix_vstack.c). Tolerance: none -- the pattern
and every value must be bit-identical (each entry sums its operands from +0.0 in
operand order, as upstream's accumulator does)."""
import ctypes as C

import numpy as np
import pytest

from sparsediff_linalg_b200._lib import matrix_p

from test_gpu_dense_ops import Lib, csr_of, pd_spec, renewed, sparse_spec, spd_spec, values_of

pytestmark = pytest.mark.gpu

vp = C.c_void_p
SIGS = {
    "new_sparse_matrix_alloc": (matrix_p, [C.c_int, C.c_int, C.c_int]),
    "sum_matrices_alloc": (None, [matrix_p, matrix_p, matrix_p]),
    "sum_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p]),
    "sum_scaled_matrices_fill_values": (None, [matrix_p, matrix_p, matrix_p, vp, vp]),
    "sum_4_matrices_alloc": (matrix_p, [matrix_p] * 4),
    "sum_4_matrices_fill_values": (None, [matrix_p] * 5),
    "sum_n_matrices_alloc": (matrix_p, [vp, C.c_int]),
    "sum_n_matrices_fill_values": (None, [vp, C.c_int, matrix_p]),
    "sum_n_matrices_fill_zero": (None, [matrix_p]),
    "sum_n_matrices_fill_add": (None, [matrix_p, C.c_int, matrix_p]),
    "vstack_matrices_alloc": (matrix_p, [vp, C.c_int]),
    "vstack_matrices_fill_values": (None, [vp, C.c_int, matrix_p]),
}


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


@pytest.fixture(scope="module")
def libs(sdl, orc):
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    out = []
    for L in (M.mlib(), orc.reference()):
        for name, (res, args) in SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        out.append(Lib(L))
    return out


def same(got, want, what):
    gp, gi, gx = csr_of(got)
    wp, wi, wx = csr_of(want)
    assert np.array_equal(gp, wp) and np.array_equal(gi, wi), what + ": pattern"
    assert np.array_equal(bits(gx), bits(wx)), what + ": values"
    assert got.contents.nnz == want.contents.nnz, what


def arr(hs):
    return (C.c_void_p * len(hs))(*[C.cast(h, C.c_void_p) for h in hs])


def _operands(rng, m, n):
    return [sparse_spec(rng, m, n, 0.15),
            pd_spec(rng, m, n, 9, 11),
            spd_spec(rng, m, n, [(5, 8), (6, 12), (1, 1)]),
            sparse_spec(rng, m, n, 0.3)]


def test_sum_two_and_scaled_match_upstream(libs):
    mine, ref = libs
    rng = np.random.default_rng(700)
    m, n = 24, 30
    specs = _operands(rng, m, n)
    for a, b in [(0, 3), (1, 0), (2, 1), (2, 2), (3, 2)]:
        hs = {}
        for name, lib in (("mine", mine), ("ref", ref)):
            A, B = lib.make(specs[a]), lib.make(specs[b])
            S = lib.L.new_sparse_matrix_alloc(m, n, A.contents.nnz + B.contents.nnz)
            lib.L.sum_matrices_alloc(A, B, S)
            lib.L.sum_matrices_fill_values(A, B, S)
            hs[name] = (A, B, S)
        same(hs["mine"][2], hs["ref"][2], f"sum {a}+{b}")
        d1 = np.ascontiguousarray(rng.uniform(-2, 2, m))
        d2 = np.ascontiguousarray(rng.uniform(-2, 2, m))
        sa, sb = renewed(specs[a], rng), renewed(specs[b], rng)
        for name, lib in (("mine", mine), ("ref", ref)):
            A, B, S = hs[name]
            Lib.set_values(A, values_of(sa))
            if b != a:
                Lib.set_values(B, values_of(sb))
            lib.L.sum_scaled_matrices_fill_values(A, B, S, d1.ctypes.data, d2.ctypes.data)
        same(hs["mine"][2], hs["ref"][2], f"scaled sum {a}+{b}")
        for name, lib in (("mine", mine), ("ref", ref)):
            lib.free(*hs[name][::-1])


def test_large_scaled_sum_matches_upstream(libs):
    """A sum of two sparse operands with 4.5M entries together: its coalescing plan
    takes the bucketed refill (factors applied while the values are bucketed)."""
    mine, ref = libs
    rng = np.random.default_rng(701)
    m, n = 3000, 3000
    specs = [sparse_spec(rng, m, n, 0.25), sparse_spec(rng, m, n, 0.25)]
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        A, B = lib.make(specs[0]), lib.make(specs[1])
        S = lib.L.new_sparse_matrix_alloc(m, n, A.contents.nnz + B.contents.nnz)
        lib.L.sum_matrices_alloc(A, B, S)
        lib.L.sum_matrices_fill_values(A, B, S)
        hs[name] = (A, B, S)
    assert hs["mine"][0].contents.nnz + hs["mine"][1].contents.nnz >= 4_194_304
    same(hs["mine"][2], hs["ref"][2], "large sum")
    d1 = np.ascontiguousarray(rng.uniform(-2, 2, m))
    d2 = np.ascontiguousarray(rng.uniform(-2, 2, m))
    for name, lib in (("mine", mine), ("ref", ref)):
        A, B, S = hs[name]
        lib.L.sum_scaled_matrices_fill_values(A, B, S, d1.ctypes.data, d2.ctypes.data)
    same(hs["mine"][2], hs["ref"][2], "large scaled sum")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])


def test_sum_4_and_sum_n_match_upstream(libs):
    mine, ref = libs
    rng = np.random.default_rng(701)
    m, n = 24, 30
    specs = _operands(rng, m, n)
    empty = ("sparse", (np.zeros(m + 1, np.int32), np.zeros(0, np.int32), np.zeros(0), m, n))
    specs.append(empty)
    order = [0, 1, 0, 4, 2, 3]     # a repeated operand and an empty one
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        H = [lib.make(sp) for sp in specs]
        S4 = lib.L.sum_4_matrices_alloc(H[0], H[1], H[2], H[3])
        lib.L.sum_4_matrices_fill_values(H[0], H[1], H[2], H[3], S4)
        ops = arr([H[k] for k in order])
        Sn = lib.L.sum_n_matrices_alloc(ops, len(order))
        lib.L.sum_n_matrices_fill_values(ops, len(order), Sn)
        S1 = lib.L.sum_n_matrices_alloc(arr([H[2]]), 1)
        lib.L.sum_n_matrices_fill_values(arr([H[2]]), 1, S1)
        hs[name] = (H, S4, Sn, S1, ops)
    same(hs["mine"][1], hs["ref"][1], "sum_4")
    same(hs["mine"][2], hs["ref"][2], "sum_n n=6")
    same(hs["mine"][3], hs["ref"][3], "sum_n n=1")
    # incremental: zero, add each operand right after its values change; an operand
    # overwritten after it was added must not leak into the sum
    new = [renewed(sp, rng) for sp in specs]
    for name, lib in (("mine", mine), ("ref", ref)):
        H, S4, Sn, S1, ops = hs[name]
        lib.L.sum_n_matrices_fill_zero(Sn)
        for pos, k in enumerate(order):
            if pos == 2:                       # operand 0's second appearance: new values
                Lib.set_values(H[0], values_of(new[0]))
            lib.L.sum_n_matrices_fill_add(H[k], pos, Sn)
        Lib.set_values(H[1], -values_of(new[1]))   # after its add: must not leak in
    same(hs["mine"][2], hs["ref"][2], "sum_n incremental")
    for name, lib in (("mine", mine), ("ref", ref)):
        H, S4, Sn, S1, ops = hs[name]
        for h in (S1, Sn, S4):
            lib.L.free_matrix(h)
        lib.free(*H)


def test_vstack_matches_upstream(libs):
    mine, ref = libs
    rng = np.random.default_rng(702)
    n = 30
    specs = [sparse_spec(rng, 10, n, 0.2), pd_spec(rng, 14, n, 6, 9),
             spd_spec(rng, 20, n, [(4, 7), (9, 13), (1, 1)]), sparse_spec(rng, 7, n, 0.0)]
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        H = [lib.make(sp) for sp in specs]
        V = lib.L.vstack_matrices_alloc(arr(H), len(H))
        v0 = V.contents.values_version
        lib.L.vstack_matrices_fill_values(arr(H), len(H), V)
        hs[name] = (H, V, V.contents.values_version - v0)
    same(hs["mine"][1], hs["ref"][1], "vstack")
    assert hs["mine"][2] == hs["ref"][2] == 1
    # change one operand: only it is recopied; nothing changed: no version bump
    new2 = renewed(specs[2], rng)
    for name, lib in (("mine", mine), ("ref", ref)):
        H, V, _ = hs[name]
        Lib.set_values(H[2], values_of(new2))
        lib.L.vstack_matrices_fill_values(arr(H), len(H), V)
        v1 = V.contents.values_version
        lib.L.vstack_matrices_fill_values(arr(H), len(H), V)
        assert V.contents.values_version == v1
    same(hs["mine"][1], hs["ref"][1], "vstack refill")
    # C written directly: the next fill recopies every operand
    for name, lib in (("mine", mine), ("ref", ref)):
        H, V, _ = hs[name]
        Lib.set_values(V, np.full(V.contents.nnz, 7.0))
        lib.L.vstack_matrices_fill_values(arr(H), len(H), V)
    same(hs["mine"][1], hs["ref"][1], "vstack after a direct write")
    for name, lib in (("mine", mine), ("ref", ref)):
        H, V, _ = hs[name]
        lib.L.free_matrix(V)
        lib.free(*H)
