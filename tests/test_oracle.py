"""The CPU oracle, pinned: against upstream's own known-answer vectors and against
the upstream library compiled from its sources (bit for bit). No GPU needed."""
import ctypes as C

import numpy as np
import pytest

import golden_vectors as gv
from sparsediff_linalg_b200 import workloads as wl
from sparsediff_linalg_b200.host import HostCSC, HostCSR, csr_from_ptr


def _csc_as_rows(A_csc):
    """Columns of a CSC = rows of L for B^T D A."""
    p, i, x, m, n = A_csc
    return np.array(p, np.int32), np.array(i, np.int32), np.array(x, float), n


def test_golden_btda(orc):
    g = gv.BTDA_SMALL
    A = gv.csc_to_csr(*g["A_csc"])
    Lp, Li, Lx, Lm = _csc_as_rows(g["B_csc"])
    Cp, Ci, Cx = orc.gustavson(Lp, Li, Lx, Lm, 1, np.array(g["d"], float), A[0], A[1], A[2], A[3], A[4])
    assert Cp.tolist() == g["Cp"] and Ci.tolist() == g["Ci"] and gv.close(Cx, g["Cx"])


@pytest.mark.parametrize("case", [gv.ATA_RANDOM, gv.ATA_RANDOM2])
def test_golden_atda(orc, case):
    A = gv.csc_to_csr(*case["A_csc"])
    Lp, Li, Lx, Lm = _csc_as_rows(case["A_csc"])
    Cp, Ci, Cx = orc.gustavson(Lp, Li, Lx, Lm, 1, np.array(case["d"], float), A[0], A[1], A[2],
                               A[3], A[4])
    assert Cp.tolist() == case["Cp"] and Ci.tolist() == case["Ci"] and gv.close(Cx, case["Cx"])


@pytest.mark.parametrize("case", [gv.ATA_SIMPLE, gv.ATA_DIAGONAL_LIKE])
def test_golden_ata_structure(orc, case):
    A = gv.csc_to_csr(*case["A_csc"])
    Lp, Li, Lx, Lm = _csc_as_rows(case["A_csc"])
    Cp, Ci, _ = orc.gustavson(Lp, Li, None, Lm, 1, None, A[0], A[1], None, A[3], A[4])
    assert Cp.tolist() == case["Cp"] and Ci.tolist() == case["Ci"]


def test_golden_conversions(orc):
    g = gv.CSR_TO_CSC
    p, i, x, m, n = g["A_csr"]
    Tp, Ti, Tx = orc.transpose(p, i, x, m, n)
    assert Tp.tolist() == g["Cp"] and Ti.tolist() == g["Ci"] and gv.close(Tx, g["Cx"])
    g = gv.CSC_TO_CSR
    p, i, x, m, n = g["A_csc"]
    Tp, Ti, Tx = orc.transpose(p, i, x, n, m)
    assert Tp.tolist() == g["Cp"] and Ti.tolist() == g["Ci"] and gv.close(Tx, g["Cx"])
    p, i, x, m, n = gv.ROUNDTRIP["A_csr"]
    Tp, Ti, Tx = orc.transpose(p, i, x, m, n)
    Rp, Ri, Rx = orc.transpose(Tp, Ti, Tx, n, m)
    assert Rp.tolist() == p and Ri.tolist() == i and Rx.tolist() == x


# ------------------------------------------------------------ port vs upstream
need_ref = pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["x"]).reference_available(),
    reason="upstream library not built")


def _ref_btda(ref, A, B_csr, d):
    """C = B^T D A by the upstream library (BTA_alloc / BTDA_fill_values)."""
    Bp, Bi, Bx, mB, nB = B_csr
    Hb = HostCSR(Bp, Bi, Bx, mB, nB)
    iw = np.zeros(max(1, nB), np.int32)
    Bc = ref.csr_to_csc_alloc(Hb.ref, iw.ctypes.data_as(C.POINTER(C.c_int)))
    ref.csr_to_csc_fill_values(Hb.ref, Bc, iw.ctypes.data_as(C.POINTER(C.c_int)))
    Ha = HostCSR(*A)
    Cm = ref.BTA_alloc(Ha.ref, Bc)
    acc = np.zeros(max(1, A[4]), float)
    dd = None if d is None else np.ascontiguousarray(d, float)
    ref.BTDA_fill_values(Ha.ref, Bc, None if dd is None else dd.ctypes.data, acc.ctypes.data, Cm)
    out = csr_from_ptr(Cm)
    ref.free_CSR_matrix(Cm)
    ref.free_CSC_matrix(Bc)
    return out


def _ref_spgemm(ref, A, B):
    """C = A B by the upstream library: A's CSR read as a CSC is A^T, so
    BTA_alloc(B, A^T as CSC) = A B (upstream matmul_dispatchers.c:147-156)."""
    Ap, Ai, Ax, mA, nA = A
    Hat = HostCSC(Ap, Ai, Ax, nA, mA)
    Hb = HostCSR(*B)
    Cm = ref.BTA_alloc(Hb.ref, Hat.ref)
    acc = np.zeros(max(1, B[4]), float)
    ref.BTDA_fill_values(Hb.ref, Hat.ref, None, acc.ctypes.data, Cm)
    out = csr_from_ptr(Cm)
    ref.free_CSR_matrix(Cm)
    return out


@need_ref
@pytest.mark.parametrize("m,nA,nB,dens,use_d", [(50, 40, 30, 0.1, True), (200, 300, 120, 0.02, True),
                                                (120, 80, 90, 0.3, False), (1, 5, 5, 1.0, True),
                                                (30, 1, 1, 0.5, True), (40, 30, 20, 0.0, True)])
def test_port_btda_matches_upstream(orc, m, nA, nB, dens, use_d):
    rng = np.random.default_rng(m * 7 + nA)
    A = wl.small_random_csr(m, nA, dens, rng)
    B = wl.small_random_csr(m, nB, dens, rng)
    d = rng.uniform(0.1, 10, m) if use_d else None
    ref = orc.reference()
    rp, ri, rx, _, _ = _ref_btda(ref, A, B, d)
    pp, pi, px = orc.btda(A, B, d)
    assert np.array_equal(rp, pp) and np.array_equal(ri, pi)
    assert np.array_equal(rx.view(np.int64), px.view(np.int64)), "values must be bit-identical"


@need_ref
def test_port_spgemm_config1_matches_upstream(orc):
    A, B = wl.spgemm_small(seed=0)
    ref = orc.reference()
    rp, ri, rx, _, _ = _ref_spgemm(ref, A, B)
    pp, pi, px = orc.spgemm(A, B)
    assert np.array_equal(rp, pp) and np.array_equal(ri, pi)
    assert np.array_equal(rx.view(np.int64), px.view(np.int64))


@need_ref
@pytest.mark.parametrize("m,n,dens", [(60, 70, 0.1), (5, 200, 0.5), (300, 10, 0.3)])
def test_port_transpose_matches_upstream(orc, m, n, dens):
    rng = np.random.default_rng(m + n)
    p, i, x, _, _ = wl.small_random_csr(m, n, dens, rng)
    ref = orc.reference()
    H = HostCSR(p, i, x, m, n)
    iw = np.zeros(max(1, n), np.int32)
    T = ref.transpose(H.ref, iw.ctypes.data_as(C.POINTER(C.c_int)))
    rp, ri, rx, _, _ = csr_from_ptr(T)
    ref.free_CSR_matrix(T)
    tp, ti, tx = orc.transpose(p, i, x, m, n)
    assert np.array_equal(rp, tp) and np.array_equal(ri, ti) and np.array_equal(rx, tx)


def _ref_row_reduce(ref, A, group, m_out):
    """Upstream row_reduce through the sparse kind's vtable slots (matrix.h:55-62)."""
    from sparsediff_linalg_b200._lib import matrix, matrix_p
    p, i, x, m, n = A
    Csr = ref.new_CSR_matrix(m, n, len(i))
    s = Csr.contents
    np.ctypeslib.as_array(s.p, shape=(m + 1,))[:] = p
    if len(i):
        np.ctypeslib.as_array(s.i, shape=(len(i),))[:] = i
        np.ctypeslib.as_array(s.x, shape=(len(i),))[:] = x
    M = ref.new_sparse_matrix(Csr)
    alloc_t = C.CFUNCTYPE(matrix_p, matrix_p, C.POINTER(C.c_int), C.c_int)
    fill_t = C.CFUNCTYPE(None, matrix_p, matrix_p)
    g = np.ascontiguousarray(group, np.int32)
    out = alloc_t(M.contents.row_reduce_alloc)(M, g.ctypes.data_as(C.POINTER(C.c_int)), m_out)
    fill_t(M.contents.row_reduce_fill_values)(M, out)
    to_csr = C.CFUNCTYPE(C.POINTER(__import__("sparsediff_linalg_b200._lib", fromlist=["x"]).CSR_matrix),
                         matrix_p)(out.contents.to_csr)
    res = csr_from_ptr(to_csr(out))
    ref.free_matrix(out)
    ref.free_matrix(M)
    return res


@need_ref
@pytest.mark.parametrize("m,n,m_out", [(80, 50, 10), (40, 30, 40), (100, 20, 1)])
def test_port_row_reduce_matches_upstream(orc, m, n, m_out):
    rng = np.random.default_rng(m * 3 + m_out)
    A = wl.small_random_csr(m, n, 0.2, rng)
    group = rng.integers(0, m_out, m)
    rp, ri, rx, _, _ = _ref_row_reduce(orc.reference(), A, group, m_out)
    pp, pi, px = orc.row_reduce(A[0], A[1], A[2], m, n, group, m_out)
    assert np.array_equal(rp, pp) and np.array_equal(ri, pi)
    assert np.array_equal(rx.view(np.int64), px.view(np.int64))


@need_ref
def test_port_coalesce_is_upstream_row_reduce(orc):
    """Coalescing == upstream row_reduce of the one-triplet-per-row CSR."""
    rng = np.random.default_rng(9)
    m, n, N = 30, 25, 400
    rows = rng.integers(0, m, N)
    cols = rng.integers(0, n, N)
    x = rng.standard_normal(N)
    x[::7] = -0.0
    A = (np.arange(N + 1, dtype=np.int32), cols.astype(np.int32), x, N, n)
    rp, ri, rx, _, _ = _ref_row_reduce(orc.reference(), A, rows, m)
    pp, pi, px = orc.coalesce(rows, cols, x, m, n)
    assert np.array_equal(rp, pp) and np.array_equal(ri, pi)
    assert np.array_equal(rx.view(np.int64), px.view(np.int64))


def test_port_kron_blocks_vs_explicit(orc):
    """blocks > 1: C = kron(I_p, L) D A equals the product with the explicit
    block-diagonal L (upstream tests/test_linalg_sparse_matmuls.h:583-588)."""
    rng = np.random.default_rng(5)
    p_blocks, nL, mL, n = 3, 7, 5, 9
    Lp, Li, Lx, _, _ = wl.small_random_csr(mL, nL, 0.4, rng)
    A = wl.small_random_csr(p_blocks * nL, n, 0.3, rng)
    d = rng.uniform(0.5, 2, p_blocks * nL)
    Cp, Ci, Cx = orc.gustavson(Lp, Li, Lx, mL, p_blocks, d, A[0], A[1], A[2], A[3], A[4])
    # explicit block-diagonal L
    rows_p, rows_i, rows_x = [0], [], []
    for b in range(p_blocks):
        for r in range(mL):
            s, e = Lp[r], Lp[r + 1]
            rows_i.extend((Li[s:e] + b * nL).tolist())
            rows_x.extend(Lx[s:e].tolist())
            rows_p.append(len(rows_i))
    Ep, Ei, Ex = orc.gustavson(rows_p, rows_i, rows_x, p_blocks * mL, 1, d, A[0], A[1], A[2], A[3], A[4])
    assert np.array_equal(Cp, Ep) and np.array_equal(Ci, Ei) and np.array_equal(Cx, Ex)


# ---------------------------------------------------------------- parallel drivers
def test_parallel_spgemm_and_btda_equal_one_call(orc):
    """Row-range pieces on a thread pool concatenate to the one-call result, bit
    for bit (incl. empty rows and rows of very different weight)."""
    from oracle import parallel
    rng = np.random.default_rng(77)
    lens = rng.integers(0, 30, 400)
    lens[::50] = 0
    lens[7] = 300
    A = wl.variable_rowlen_csr(400, 500, lens, rng)
    B = wl.small_random_csr(500, 300, 0.02, rng)
    want = orc.spgemm(A, B)
    got = parallel.spgemm(A, B, threads=3)
    assert parallel.compare_csr(got, want)["bit_identical"]
    A2 = wl.small_random_csr(500, 200, 0.03, rng)
    d = rng.uniform(0.1, 10, 500)
    want = orc.btda(A2, B, d)
    got = parallel.btda(A2, B, d, threads=4)
    r = parallel.compare_csr(got, want)
    assert r["structure_equal"] and r["bit_identical"] and r["max_rel_err"] == 0.0


def test_parallel_coalesce_equals_one_call(orc):
    from oracle import parallel
    rng = np.random.default_rng(78)
    m, n, N = 300, 200, 20000
    rows = rng.integers(0, m, N).astype(np.int32)
    rows[rows == 5] = 6                                     # an empty output row
    cols = rng.integers(0, n, N).astype(np.int32)
    x = rng.standard_normal(N)
    x[::11] = -0.0
    want = orc.coalesce(rows, cols, x, m, n)
    got = parallel.coalesce(rows, cols, x, m, n, threads=5)
    assert parallel.compare_csr(got, want)["bit_identical"]


def test_compare_csr_reports_errors(orc):
    from oracle import parallel
    p = np.array([0, 2, 3], np.int32)
    i = np.array([0, 3, 1], np.int32)
    x = np.array([1.0, -2.0, 0.5])
    r = parallel.compare_csr((p, i, x), (p, i, x.copy()))
    assert r["bit_identical"] and r["max_rel_err"] == 0.0
    y = x.copy()
    y[1] *= 1 + 2e-13
    r = parallel.compare_csr((p, i, y), (p, i, x))
    assert r["structure_equal"] and not r["bit_identical"] and 1e-13 < r["max_rel_err"] < 1e-12
    assert r["within_tol"]
    r = parallel.compare_csr((p, np.array([0, 2, 1], np.int32), x), (p, i, x))
    assert not r["structure_equal"]


def _blocks_csr_by_loops(blocks, Sp, Si, Sx):
    """The definition, term by term: per block, output columns the union of S's rows
    in col_perm (ascending); each cell summed from +0.0 over rows r ascending."""
    out = []
    for X, cperm in blocks:
        ents = [(int(Si[q]), r, float(Sx[q])) for r, row in enumerate(cperm)
                for q in range(Sp[row], Sp[row + 1])]
        cols = sorted({c for c, _, _ in ents})
        loc = {c: k for k, c in enumerate(cols)}
        C = np.zeros((X.shape[0], len(cols)))
        for i in range(X.shape[0]):
            for c, r, v in ents:
                C[i, loc[c]] = C[i, loc[c]] + X[i, r] * v
        out.append((np.array(cols, np.int32), C))
    return out


def test_blocks_csr_oracle_matches_definition(orc):
    rng = np.random.default_rng(79)
    S = wl.small_random_csr(40, 60, 0.1, rng)
    blocks = [(rng.standard_normal((5, 12)), np.sort(rng.choice(40, 12, replace=False)).astype(np.int32))
              for _ in range(3)]
    blocks.append((rng.standard_normal((3, 12)), blocks[0][1]))   # a repeated col_perm
    blocks.append((rng.standard_normal((2, 1)), np.array([7], np.int32)))
    want = _blocks_csr_by_loops(blocks, S[0], S[1], S[2])
    got = orc.blocks_csr(blocks, S[0], S[1], S[2], 60)
    for (gc, gv_), (wc, wv) in zip(got, want):
        assert np.array_equal(gc, wc)
        assert np.array_equal(gv_.view(np.int64), wv.view(np.int64))


@need_ref
def test_blocks_csr_oracle_matches_upstream_pd(orc):
    """One permuted_dense block times a sparse matrix by the upstream library
    (BA_matrices_* with B permuted_dense, src/permuted_dense/permuted_dense_linalg.c:313-430)
    against the oracle's dense-block product, bit for bit."""
    from sparsediff_linalg_b200._lib import CSR_p, matrix_p
    ref = orc.reference()
    rng = np.random.default_rng(80)
    A = wl.small_random_csr(90, 400, 0.04, rng)            # S: 90 x 400
    rp = np.sort(rng.choice(150, size=21, replace=False)).astype(np.int32)
    cp = np.sort(rng.choice(90, size=33, replace=False)).astype(np.int32)
    X = rng.standard_normal((21, 33))
    c = ref.new_CSR_matrix(90, 400, len(A[1]))
    s = c.contents
    np.ctypeslib.as_array(s.p, shape=(91,))[:] = A[0]
    np.ctypeslib.as_array(s.i, shape=(max(1, len(A[1])),))[:len(A[1])] = A[1]
    np.ctypeslib.as_array(s.x, shape=(max(1, len(A[1])),))[:len(A[1])] = A[2]
    Ar = ref.new_sparse_matrix(c)
    Br = ref.new_permuted_dense(150, 90, 21, 33, rp.ctypes.data, cp.ctypes.data, X.ctypes.data)
    Cr = ref.BA_matrices_alloc(Br, Ar)
    ref.BA_matrices_fill_values(Br, Ar, Cr)
    to_csr = C.CFUNCTYPE(CSR_p, matrix_p)
    wp, wi, wx, wm, wn = csr_from_ptr(to_csr(Cr.contents.to_csr)(Cr))
    (cols, Ck), = orc.blocks_csr([(X, cp)], A[0], A[1], A[2], 400)
    for k, r in enumerate(rp):
        assert np.array_equal(wi[wp[r]:wp[r + 1]], cols)
        assert np.array_equal(wx[wp[r]:wp[r + 1]].view(np.int64), Ck[k].view(np.int64))
    ref.free_matrix(Cr)
    ref.free_matrix(Br)
    ref.free_matrix(Ar)
