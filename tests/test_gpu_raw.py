"""GPU parity of the upstream raw entry points (BTA_alloc / BTDA_fill_values,
csr_to_csc / csc_to_csr / AT / transpose, COO coalescing) called through the C ABI
with host structs, against the CPU oracle (bit for bit) and upstream's known-answer
vectors. Tolerance: none -- structure and values must be bit-identical."""
import ctypes as C

import numpy as np
import pytest

import golden_vectors as gv
from sparsediff_linalg_b200 import workloads as wl
from sparsediff_linalg_b200.host import HostCOO, HostCSC, HostCSR, csr_from_ptr

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


def assert_same(got, want):
    gp, gi, gx = got[:3]
    wp, wi, wx = want[:3]
    assert np.array_equal(gp, wp), "row offsets differ"
    assert np.array_equal(gi, wi), "column indices differ"
    assert np.array_equal(bits(gx), bits(wx)), \
        f"values differ (max abs diff {np.max(np.abs(np.asarray(gx) - np.asarray(wx)), initial=0)})"


def gpu_btda(L, A, B_csr, d, refills=()):
    """C = B^T D A through csr_to_csc + BTA_alloc + BTDA_fill_values."""
    Hb = HostCSR(*B_csr)
    Bc = L.csr_to_csc_alloc(Hb.ref, None)
    assert Bc, L.sdl_last_error()
    L.csr_to_csc_fill_values(Hb.ref, Bc, None)
    Ha = HostCSR(*A)
    Cm = L.BTA_alloc(Ha.ref, Bc)
    assert Cm, L.sdl_last_error()
    dd = None if d is None else np.ascontiguousarray(d, float)
    L.BTDA_fill_values(Ha.ref, Bc, None if dd is None else dd.ctypes.data, None, Cm)
    out = [csr_from_ptr(Cm)]
    for (ax, bx, dn) in refills:
        Ha.set_values(ax)
        Hb.set_values(bx)
        L.csr_to_csc_fill_values(Hb.ref, Bc, None)
        dd = None if dn is None else np.ascontiguousarray(dn, float)
        L.BTDA_fill_values(Ha.ref, Bc, None if dd is None else dd.ctypes.data, None, Cm)
        out.append(csr_from_ptr(Cm))
    L.free_CSR_matrix(Cm)
    L.free_CSC_matrix(Bc)
    return out


def test_golden_btda(sdl):
    g = gv.BTDA_SMALL
    A = gv.csc_to_csr(*g["A_csc"])
    Hb = HostCSC(*g["B_csc"])
    Ha = HostCSR(*A)
    Cm = sdl.BTA_alloc(Ha.ref, Hb.ref)
    d = np.array(g["d"], float)
    sdl.BTDA_fill_values(Ha.ref, Hb.ref, d.ctypes.data, None, Cm)
    p, i, x, m, n = csr_from_ptr(Cm)
    sdl.free_CSR_matrix(Cm)
    assert p.tolist() == g["Cp"] and i.tolist() == g["Ci"] and x.tolist() == g["Cx"]
    assert (m, n) == (2, 3)


@pytest.mark.parametrize("case", [gv.ATA_RANDOM, gv.ATA_RANDOM2])
def test_golden_atda(sdl, orc, case):
    A = gv.csc_to_csr(*case["A_csc"])
    Hc = HostCSC(*case["A_csc"])
    Ha = HostCSR(*A)
    Cm = sdl.BTA_alloc(Ha.ref, Hc.ref)
    d = np.array(case["d"], float)
    sdl.BTDA_fill_values(Ha.ref, Hc.ref, d.ctypes.data, None, Cm)
    got = csr_from_ptr(Cm)
    sdl.free_CSR_matrix(Cm)
    assert got[0].tolist() == case["Cp"] and got[1].tolist() == case["Ci"]
    assert gv.close(got[2], case["Cx"])
    p, i, x, m, n = case["A_csc"]
    want = orc.gustavson(p, i, x, n, 1, d, A[0], A[1], A[2], A[3], A[4])
    assert_same(got, want)


@pytest.mark.parametrize("m,nA,nB,dens,use_d", [
    (50, 40, 30, 0.1, True), (200, 300, 120, 0.02, True), (120, 80, 90, 0.3, False),
    (1, 5, 5, 1.0, True), (30, 1, 1, 0.5, True), (40, 30, 20, 0.0, True),
    (3000, 2000, 1500, 0.004, True)])
def test_btda_random_bit_exact(sdl, orc, m, nA, nB, dens, use_d):
    rng = np.random.default_rng(m * 7 + nA)
    A = wl.small_random_csr(m, nA, dens, rng)
    B = wl.small_random_csr(m, nB, dens, rng)
    d = rng.uniform(0.1, 10, m) if use_d else None
    refill = (rng.standard_normal(len(A[1])), rng.standard_normal(len(B[1])),
              rng.uniform(0.1, 10, m) if use_d else None)
    got = gpu_btda(sdl, A, B, d, refills=[refill])
    assert_same(got[0], orc.btda(A, B, d))
    A2 = (A[0], A[1], refill[0], A[3], A[4])
    B2 = (B[0], B[1], refill[1], B[3], B[4])
    assert_same(got[1], orc.btda(A2, B2, refill[2]))


def _skewed_operands(rng, m, nA, nB, col_lens, row_len):
    """B with prescribed column lengths (rows of L) and A with row_len entries per
    row: row r of C has ~col_lens[r] * row_len terms, spanning every kernel class."""
    cols = []
    for c, ln in enumerate(col_lens):
        rows = rng.choice(m, size=min(ln, m), replace=False)
        cols.append(np.stack([rows, np.full(len(rows), c)], 1))
    ent = np.concatenate(cols)
    order = np.lexsort((ent[:, 1], ent[:, 0]))
    ent = ent[order]
    Bp = np.zeros(m + 1, np.int32)
    np.add.at(Bp, ent[:, 0] + 1, 1)
    Bp = np.cumsum(Bp).astype(np.int32)
    B = (Bp, ent[:, 1].astype(np.int32), rng.standard_normal(len(ent)), m, nB)
    A = wl.fixed_rowlen_csr(m, nA, row_len, rng)
    return A, B


def test_btda_every_row_class(sdl, orc):
    """Rows from 0 to ~120k terms: warp classes (<=32/128/512), CTA classes (2k/8k
    entries), the bitmap symbolic class and the global-accumulator numeric class."""
    rng = np.random.default_rng(77)
    m, nA = 6000, 30000
    col_lens = [0, 1, 2, 3, 5, 8, 15, 30, 60, 100, 200, 400, 800, 1500, 3000, 6000] + [4] * 200
    A, B = _skewed_operands(rng, m, nA, len(col_lens), col_lens, 20)
    d = rng.uniform(0.1, 10, m)
    got = gpu_btda(sdl, A, B, d)
    assert_same(got[0], orc.btda(A, B, d))


def test_btda_many_collisions(sdl, orc):
    """Few distinct columns: every output entry collects many terms, which stresses
    the in-order application of same-entry terms inside a chunk."""
    rng = np.random.default_rng(78)
    m, nA = 4000, 12
    A = wl.fixed_rowlen_csr(m, nA, 6, rng)
    col_lens = [1, 5, 40, 300, 1000, 4000]
    _, B = _skewed_operands(rng, m, nA, len(col_lens), col_lens, 6)
    d = rng.uniform(0.1, 10, m)
    got = gpu_btda(sdl, A, B, d)
    assert_same(got[0], orc.btda(A, B, d))


def test_btda_tile_outputs_with_long_term_lists(sdl, orc):
    """Tile rows whose outputs collect 2 to ~70 terms (every list length modulo the
    kernel's batch of 4), with values spread over 16 decades so that a change of
    summation order would show in the bits; thousands of tiles, so the refill's
    pipeline runs in steady state and wraps its buffers many times."""
    rng = np.random.default_rng(79)
    m, nA = 60000, 4
    A = wl.fixed_rowlen_csr(m, nA, 4, rng)          # every A row hits all 4 columns
    A = (A[0], A[1], A[2] * 10.0 ** rng.integers(-8, 9, len(A[2])), A[3], A[4])
    col_lens = list(rng.integers(1, 72, 6000))      # rows of L: 1..71 entries
    _, B = _skewed_operands(rng, m, nA, len(col_lens), col_lens, 4)
    d = rng.uniform(0.1, 10, m)
    got = gpu_btda(sdl, A, B, d)
    assert_same(got[0], orc.btda(A, B, d))


def test_spgemm_config1_bit_exact(sdl, orc):
    """C = A B for the 2000 x 2000, 5 per row case: A's CSR read as CSC is A^T."""
    A, B = wl.spgemm_small(seed=0)
    Hat = HostCSC(A[0], A[1], A[2], A[4], A[3])
    Hb = HostCSR(*B)
    Cm = sdl.BTA_alloc(Hb.ref, Hat.ref)
    sdl.BTDA_fill_values(Hb.ref, Hat.ref, None, None, Cm)
    got = csr_from_ptr(Cm)
    sdl.free_CSR_matrix(Cm)
    assert_same(got, orc.spgemm(A, B))


# ------------------------------------------------------------ conversions
def test_golden_conversions(sdl):
    g = gv.CSR_TO_CSC
    H = HostCSR(*g["A_csr"])
    Cc = sdl.csr_to_csc_alloc(H.ref, None)
    sdl.csr_to_csc_fill_values(H.ref, Cc, None)
    p, i, x, _, _ = csr_from_ptr(Cc, rows_attr="n")
    sdl.free_CSC_matrix(Cc)
    assert p.tolist() == g["Cp"] and i.tolist() == g["Ci"] and x.tolist() == g["Cx"]
    g = gv.CSC_TO_CSR
    H = HostCSC(*g["A_csc"])
    Cr = sdl.csc_to_csr_alloc(H.ref, None)
    sdl.csc_to_csr_fill_values(H.ref, Cr, None)
    p, i, x, _, _ = csr_from_ptr(Cr)
    sdl.free_CSR_matrix(Cr)
    assert p.tolist() == g["Cp"] and i.tolist() == g["Ci"] and x.tolist() == g["Cx"]
    p0, i0, x0, m, n = gv.ROUNDTRIP["A_csr"]
    H = HostCSR(p0, i0, x0, m, n)
    Cc = sdl.csr_to_csc_alloc(H.ref, None)
    sdl.csr_to_csc_fill_values(H.ref, Cc, None)
    Cr = sdl.csc_to_csr_alloc(Cc, None)
    sdl.csc_to_csr_fill_values(Cc, Cr, None)
    p, i, x, _, _ = csr_from_ptr(Cr)
    sdl.free_CSR_matrix(Cr)
    sdl.free_CSC_matrix(Cc)
    assert p.tolist() == p0 and i.tolist() == i0 and x.tolist() == x0


@pytest.mark.parametrize("m,n,dens", [(60, 70, 0.1), (5, 200, 0.5), (300, 10, 0.3), (0, 5, 0.1),
                                      (7, 0, 0.1), (2000, 3000, 0.002)])
def test_transpose_bit_exact(sdl, orc, m, n, dens):
    rng = np.random.default_rng(m + n)
    p, i, x, _, _ = wl.small_random_csr(m, n, dens, rng)
    H = HostCSR(p, i, x, m, n)
    T = sdl.transpose(H.ref, None)
    got = csr_from_ptr(T)
    sdl.free_CSR_matrix(T)
    assert_same(got, orc.transpose(p, i, x, m, n))
    # AT_alloc + AT_fill_values with new values
    x2 = rng.standard_normal(len(i))
    H.set_values(x2)
    AT = sdl.AT_alloc(H.ref, None)
    sdl.AT_fill_values(H.ref, AT, None)
    got = csr_from_ptr(AT)
    sdl.free_CSR_matrix(AT)
    assert_same(got, orc.transpose(p, i, x2, m, n))


def test_transpose_long_segments(sdl, orc):
    """Dense columns (long output segments: warp, CTA and merge-sort classes) and
    unsorted rows with duplicate columns (order follows source position)."""
    rng = np.random.default_rng(11)
    m, n = 30000, 40
    rows = []
    for r in range(m):
        k = rng.integers(1, 6)
        c = rng.integers(0, n, k)
        c[0] = 0                     # column 0 is dense: a 30000-long segment
        if r % 3 == 0:
            c = np.append(c, 1)      # column 1: ~10000 entries
        rows.append(c)
    p = np.zeros(m + 1, np.int32)
    p[1:] = np.cumsum([len(c) for c in rows])
    i = np.concatenate(rows).astype(np.int32)
    x = rng.standard_normal(len(i))
    H = HostCSR(p, i, x, m, n)
    Cc = sdl.csr_to_csc_alloc(H.ref, None)
    sdl.csr_to_csc_fill_values(H.ref, Cc, None)
    got = csr_from_ptr(Cc, rows_attr="n")
    sdl.free_CSC_matrix(Cc)
    assert_same(got, orc.transpose(p, i, x, m, n))


# ------------------------------------------------------------ coalesce
@pytest.mark.parametrize("m,n,N", [(30, 25, 400), (1, 1, 50), (100, 1000, 5000), (50, 7, 0),
                                   (2000, 3000, 200000)])
def test_coalesce_bit_exact(sdl, orc, m, n, N):
    rng = np.random.default_rng(N + m)
    rows = rng.integers(0, m, N).astype(np.int32)
    cols = rng.integers(0, n, N).astype(np.int32)
    x = rng.standard_normal(N)
    x[::5] = -0.0
    H = HostCOO(rows, cols, x, m, n)
    Cm = sdl.COO_coalesce_alloc(H.ref)
    assert Cm, sdl.sdl_last_error()
    sdl.COO_coalesce_fill_values(H.ref, Cm)
    got = csr_from_ptr(Cm)
    want = orc.coalesce(rows, cols, x, m, n)
    assert_same(got, want)
    # refill with new values
    x2 = rng.standard_normal(N)
    H.x[...] = x2
    sdl.COO_coalesce_fill_values(H.ref, Cm)
    got = csr_from_ptr(Cm)
    sdl.free_CSR_matrix(Cm)
    assert_same(got, orc.coalesce(rows, cols, x2, m, n))


@pytest.mark.parametrize("m,n,N,neg_zero", [(2000, 2000, 5_000_000, True),     # ~3.7M outputs, many buckets
                                             (300, 300, 4_500_000, False),       # 90k outputs, ~50 terms each
                                             (100_000, 100_000, 4_194_304, True)])  # exactly the threshold
def test_coalesce_bucketed_refill_bit_exact(sdl, orc, m, n, N, neg_zero):
    """Inputs of at least 4Mi triplets take the bucketed refill (values first written
    into output-range buckets, then summed per output from L2): the same bits as
    the oracle, on the first fill and on a refill with new values."""
    from oracle import parallel
    rng = np.random.default_rng(N % 1000 + m)
    rows = rng.integers(0, m, N).astype(np.int32)
    cols = rng.integers(0, n, N).astype(np.int32)
    x = rng.standard_normal(N)
    if neg_zero:
        x[::7] = -0.0
    H = HostCOO(rows, cols, x, m, n)
    Cm = sdl.COO_coalesce_alloc(H.ref)
    assert Cm, sdl.sdl_last_error()
    for rnd in range(2):
        sdl.COO_coalesce_fill_values(H.ref, Cm)
        got = csr_from_ptr(Cm)
        want = parallel.coalesce(rows, cols, H.x.copy(), m, n)
        assert_same(got, want)
        H.x[...] = rng.standard_normal(N)
    sdl.free_CSR_matrix(Cm)


def test_fills_make_no_device_allocation(sdl):
    rng = np.random.default_rng(3)
    A = wl.small_random_csr(500, 400, 0.02, rng)
    B = wl.small_random_csr(500, 300, 0.02, rng)
    Hb = HostCSR(*B)
    Bc = sdl.csr_to_csc_alloc(Hb.ref, None)
    Ha = HostCSR(*A)
    Cm = sdl.BTA_alloc(Ha.ref, Bc)
    d = rng.uniform(0.1, 10, 500)
    sdl.csr_to_csc_fill_values(Hb.ref, Bc, None)
    sdl.BTDA_fill_values(Ha.ref, Bc, d.ctypes.data, None, Cm)
    before = sdl.sdl_device_alloc_count()
    for _ in range(3):
        sdl.csr_to_csc_fill_values(Hb.ref, Bc, None)
        sdl.BTDA_fill_values(Ha.ref, Bc, d.ctypes.data, None, Cm)
    assert sdl.sdl_device_alloc_count() == before
    sdl.free_CSR_matrix(Cm)
    sdl.free_CSC_matrix(Bc)


def test_invalid_input_is_rejected_not_run(sdl):
    """Out-of-range indices are caught by the device validation pass before any
    kernel indexes with them; status mode returns NULL with SDL_ERR_INVALID."""
    sdl.sdl_set_fatal_errors(0)
    try:
        H = HostCSR([0, 2], [0, 9], [1.0, 2.0], 1, 3)   # column 9 >= n = 3
        out = sdl.csr_to_csc_alloc(H.ref, None)
        assert not out
        assert sdl.sdl_last_status() == 3
    finally:
        sdl.sdl_set_fatal_errors(1)


def test_btda_signed_zeros_and_pairs(sdl, orc):
    """Entries with exactly two terms are added in either order by the fast tile
    path; with +0.0 / -0.0 / tiny values mixed in, results must still be
    bit-identical to upstream's ordered sum (0 + a) + b."""
    rng = np.random.default_rng(91)
    m, nA, nB = 3000, 400, 300
    A = wl.fixed_rowlen_csr(m, nA, 6, rng)
    B = wl.fixed_rowlen_csr(m, nB, 4, rng)
    ax = A[2].copy()
    ax[::3] = -0.0
    ax[1::7] = 0.0
    ax[2::11] = 1e-300
    bx = B[2].copy()
    bx[::5] = -0.0
    A = (A[0], A[1], ax, A[3], A[4])
    B = (B[0], B[1], bx, B[3], B[4])
    d = rng.uniform(0.1, 10, m)
    d[::13] = -0.0
    got = gpu_btda(sdl, A, B, d)
    assert_same(got[0], orc.btda(A, B, d))
