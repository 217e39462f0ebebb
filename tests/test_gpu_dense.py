"""Dense blocks times a sparse CSR on the GPU (permuted_dense / stacked_pd x sparse),
against the CPU oracle and the upstream library itself. Tolerance: none -- the
blocks' column sets and every value must be bit-identical (each output is summed
in upstream's order)."""
import ctypes as C

import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


def _blocks(rng, S_m, specs):
    """specs: [(m0, n0)]; col_perm = n0 sorted distinct rows of S."""
    out = []
    for m0, n0 in specs:
        perm = np.sort(rng.choice(S_m, size=n0, replace=False)).astype(np.int32)
        X = rng.standard_normal((m0, n0)) * 10.0 ** rng.integers(-6, 7, (m0, n0))
        out.append((X, perm))
    return out


def _run_device(blocks, S, keep_empty):
    import torch
    from sparsediff_linalg_b200.device import BlocksCsr
    Sp, Si, Sx, S_m, S_n = S
    P = BlocksCsr([X.shape[0] for X, _ in blocks], [X.shape[1] for X, _ in blocks],
                  [c for _, c in blocks], Sp, Si, S_m, S_n, keep_empty=keep_empty)
    Bv = torch.as_tensor(np.concatenate([X.ravel() for X, _ in blocks] + [np.zeros(1)]), device="cuda")
    Sx_d = torch.as_tensor(np.asarray(Sx, np.float64), device="cuda")
    Cv = torch.full((max(1, P.c_values),), np.nan, dtype=torch.float64, device="cuda")
    P.fill(Bv, Sx_d, Cv)
    torch.cuda.synchronize()
    Cv = Cv.cpu().numpy()
    res, off = [], 0
    for src, m0, n0c, perm in P.blocks:
        res.append((src, perm, Cv[off:off + m0 * n0c].reshape(m0, n0c)))
        off += m0 * n0c
    return P, res


@pytest.mark.parametrize("keep_empty", [False, True])
def test_blocks_csr_bit_exact(sdl, orc, keep_empty):
    """Blocks of many shapes (incl. 1 x 1, empty-result blocks, columns with more
    than 8 terms) against the oracle; empty blocks dropped unless keep_empty."""
    rng = np.random.default_rng(91)
    S_m, S_n = 300, 5000
    lens = rng.integers(0, 40, S_m)
    lens[:20] = 0                       # rows of S without entries
    lens[20:25] = 3000                  # dense-ish rows: columns with many terms
    S = wl.variable_rowlen_csr(S_m, S_n, lens, rng)
    specs = [(1, 1), (7, 13), (64, 256), (33, 5), (5, 40), (16, 300)]
    blocks = _blocks(rng, S_m, specs)
    blocks.append((rng.standard_normal((4, 10)), np.arange(10, dtype=np.int32)))  # only empty rows
    want = orc.blocks_csr(blocks, S[0], S[1], S[2], S_n)
    P, got = _run_device(blocks, S, keep_empty)
    kept = [k for k, (cols, C_k) in enumerate(want) if keep_empty or C_k.size]
    assert [g[0] for g in got] == kept
    for (src, perm, Cg) in got:
        cols, Cw = want[src]
        assert np.array_equal(perm, cols)
        assert np.array_equal(bits(Cg), bits(Cw)), f"block {src}"


def test_blocks_csr_config_shape(sdl, orc):
    """The 64 x 256 block shape of the benchmark (S 256 x 20000, 6 entries per
    column), four blocks."""
    rng = np.random.default_rng(92)
    S_m, S_n = 256, 20000
    St = wl.fixed_rowlen_csr(S_n, S_m, 6, rng)          # CSC of S as a CSR of S^T
    from oracle import oracle
    Sp, Si, Sx = oracle.transpose(St[0], St[1], St[2], S_n, S_m)
    S = (Sp, Si, Sx, S_m, S_n)
    blocks = [(rng.standard_normal((64, 256)), np.arange(256, dtype=np.int32)) for _ in range(4)]
    want = orc.blocks_csr(blocks, Sp, Si, Sx, S_n)
    P, got = _run_device(blocks, S, False)
    assert len(got) == 4
    for (src, perm, Cg) in got:
        cols, Cw = want[src]
        assert np.array_equal(perm, cols)
        assert np.array_equal(bits(Cg), bits(Cw))


@pytest.mark.parametrize("specs", [[(100, 20), (65, 7), (3, 9)], [(8, 400), (64, 30)]],
                         ids=["blocks_over_64_rows", "wide_source_block"])
def test_blocks_csr_tall_and_wide_blocks_bit_exact(sdl, orc, specs):
    """Blocks of more than 64 rows (several row passes of a tile) and a 400-column
    source block: the same bits as the oracle."""
    rng = np.random.default_rng(93)
    S_m, S_n = 500, 3000
    lens = rng.integers(0, 30, S_m)
    lens[:5] = 1500
    S = wl.variable_rowlen_csr(S_m, S_n, lens, rng)
    blocks = _blocks(rng, S_m, specs)
    want = orc.blocks_csr(blocks, S[0], S[1], S[2], S_n)
    P, got = _run_device(blocks, S, False)
    assert len(got) == len(specs)
    for (src, perm, Cg) in got:
        cols, Cw = want[src]
        assert np.array_equal(perm, cols)
        assert np.array_equal(bits(Cg), bits(Cw)), f"block {src}"


def test_blocks_csr_many_small_blocks_bit_exact(sdl, orc):
    """Forty blocks of 1 to 64 rows over few columns, some with an output narrower
    than one 32-column tile, empty ones kept."""
    rng = np.random.default_rng(94)
    S_m, S_n = 200, 900
    lens = rng.integers(0, 6, S_m)
    S = wl.variable_rowlen_csr(S_m, S_n, lens, rng)
    specs = [(int(rng.integers(1, 65)), int(rng.integers(1, 60))) for _ in range(40)]
    blocks = _blocks(rng, S_m, specs)
    want = orc.blocks_csr(blocks, S[0], S[1], S[2], S_n)
    P, got = _run_device(blocks, S, True)
    for (src, perm, Cg) in got:
        cols, Cw = want[src]
        assert np.array_equal(perm, cols)
        assert np.array_equal(bits(Cg), bits(Cw)), f"block {src}"


def test_BA_pd_sparse_matches_upstream_library(sdl, orc):
    """BA_matrices_alloc / BA_matrices_fill_values with B permuted_dense and A
    sparse, through the drop-in C ABI, against the same calls on the upstream
    library compiled from its sources; then a refill with new values of both."""
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    from sparsediff_linalg_b200._lib import CSR_p, matrix_p
    from sparsediff_linalg_b200.host import csr_from_ptr
    ref = orc.reference()
    rng = np.random.default_rng(93)
    A = wl.small_random_csr(120, 900, 0.03, rng)       # S: 120 x 900
    rp = np.sort(rng.choice(200, size=37, replace=False)).astype(np.int32)
    cp = np.sort(rng.choice(120, size=50, replace=False)).astype(np.int32)
    X = rng.standard_normal((37, 50))
    to_csr = C.CFUNCTYPE(CSR_p, matrix_p)

    def ref_sparse(csr):
        p, i, x, m, n = csr
        c = ref.new_CSR_matrix(m, n, len(i))
        s = c.contents
        np.ctypeslib.as_array(s.p, shape=(m + 1,))[:] = p
        np.ctypeslib.as_array(s.i, shape=(max(1, len(i)),))[:len(i)] = i
        np.ctypeslib.as_array(s.x, shape=(max(1, len(i)),))[:len(i)] = x
        return ref.new_sparse_matrix(c)

    Ar = ref_sparse(A)
    Br = ref.new_permuted_dense(200, 120, 37, 50, rp.ctypes.data, cp.ctypes.data, X.ctypes.data)
    Cr = ref.BA_matrices_alloc(Br, Ar)
    ref.BA_matrices_fill_values(Br, Ar, Cr)
    want = csr_from_ptr(to_csr(Cr.contents.to_csr)(Cr))

    Am = M.SparseMatrix.from_csr(*A)
    Bm = M.permuted_dense(200, 120, rp, cp, X)
    Cm = M.BA(Bm, Am)
    M.BA_fill(Bm, Am, Cm)
    got = Cm.csr()
    for g, w in zip(got, want[:3]):
        assert np.array_equal(bits(g) if g.dtype == np.float64 else g, bits(w) if w.dtype == np.float64 else w)
    # refill: new values of A and B in both libraries
    ax = rng.standard_normal(len(A[1]))
    X2 = rng.standard_normal((37, 50))
    Am.set_values(ax)
    Bm.set_values(X2.ravel())
    M.BA_fill(Bm, Am, Cm)
    np.ctypeslib.as_array(Ar.contents.x, shape=(len(ax),))[:] = ax
    Ar.contents.values_version += 1
    np.ctypeslib.as_array(Br.contents.x, shape=(X2.size,))[:] = X2.ravel()
    Br.contents.values_version += 1
    ref.BA_matrices_fill_values(Br, Ar, Cr)
    want2 = csr_from_ptr(to_csr(Cr.contents.to_csr)(Cr))
    assert np.array_equal(bits(Cm.csr()[2]), bits(want2[2]))
    ref.free_matrix(Cr)
    ref.free_matrix(Br)
    ref.free_matrix(Ar)


# ---------------------------------------------------------------- A^T D A (FP64 tensor cores)
def _spd_blocks(rng, m, n, specs):
    """Row-disjoint blocks (a stacked_pd): specs [(m0, n0)]; col_perms overlap."""
    rows = rng.permutation(m)
    out, at = [], 0
    for m0, n0 in specs:
        rp = np.sort(rows[at:at + m0]).astype(np.int32)
        at += m0
        cp = np.sort(rng.choice(n, size=n0, replace=False)).astype(np.int32)
        out.append((rng.standard_normal((m0, n0)), rp, cp))
    return out


def _close(got, want, scale, what):
    err = np.abs(got - want)
    bound = 1e-12 * scale + 1e-300
    assert np.all(err <= bound), f"{what}: max err/bound {np.max(err / bound)}"


def test_blocks_ata_matches_oracle(sdl, orc):
    """Overlapping col_perms (several signatures), uneven shapes (K not a multiple of
    4, n0 not a multiple of 16), with and without d: structure exact, values within
    1e-12 of the sum of |terms| (upstream's dgemm order is unspecified)."""
    import torch
    from sparsediff_linalg_b200.device import BlocksAta
    rng = np.random.default_rng(94)
    m, n = 400, 70
    blocks = _spd_blocks(rng, m, n, [(13, 20), (64, 45), (7, 3), (30, 70), (1, 1), (50, 33)])
    for use_d in (True, False):
        d = rng.uniform(0.1, 10, m) if use_d else None
        want = orc.blocks_ata(blocks, d, n)
        P = BlocksAta([X.shape[0] for X, _, _ in blocks], [X.shape[1] for X, _, _ in blocks],
                      [r for _, r, _ in blocks], [c for _, _, c in blocks], m, n)
        assert P.out_blocks == len(want)
        Xv = torch.as_tensor(np.concatenate([X.ravel() for X, _, _ in blocks]), device="cuda")
        dd = None if d is None else torch.as_tensor(d, device="cuda")
        Cv = torch.full((P.c_values,), np.nan, dtype=torch.float64, device="cuda")
        P.fill(Xv, dd, Cv)
        torch.cuda.synchronize()
        Cv = Cv.cpu().numpy()
        off = 0
        for (rows, cols), (wr, wc, Cw, Ca) in zip(P.blocks, want):
            assert np.array_equal(rows, wr) and np.array_equal(cols, wc)
            Cg = Cv[off:off + len(rows) * len(cols)].reshape(len(rows), len(cols))
            off += Cg.size
            _close(Cg, Cw, Ca, "A^T D A block")


def _ref_csr(ref, M):
    from sparsediff_linalg_b200._lib import CSR_p, matrix_p
    from sparsediff_linalg_b200.host import csr_from_ptr
    to_csr = C.CFUNCTYPE(CSR_p, matrix_p)
    return csr_from_ptr(to_csr(M.contents.to_csr)(M))


def test_ATDA_stacked_pd_matches_upstream_library(sdl, orc):
    """ATA_matrices_alloc / ATDA_matrices_fill_values with A stacked_pd through the
    drop-in C ABI vs the upstream library: identical structure, values within
    1e-12 of the sum of |terms|; a refill with new values and d."""
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    ref = orc.reference()
    rng = np.random.default_rng(95)
    m, n = 300, 60
    blocks = _spd_blocks(rng, m, n, [(20, 30), (64, 25), (9, 60), (40, 12)])
    d = rng.uniform(0.1, 10, m)

    def build_ref(blks):
        arr = (C.c_void_p * len(blks))()
        for k, (X, rp, cp) in enumerate(blks):
            Xc = np.ascontiguousarray(X)
            pm = ref.new_permuted_dense(m, n, len(rp), len(cp), rp.ctypes.data, cp.ctypes.data, Xc.ctypes.data)
            arr[k] = C.cast(pm, C.c_void_p)
        return ref.new_stacked_pd(m, n, len(blks), arr, None, None)

    Ar = build_ref(blocks)
    Cr = ref.ATA_matrices_alloc(Ar)
    ref.ATDA_matrices_fill_values(Ar, d.ctypes.data, Cr)
    wp, wi, wx = _ref_csr(ref, Cr)[:3]

    Am = M.stacked_pd(m, n, [M.permuted_dense(m, n, rp, cp, X) for X, rp, cp in blocks])
    Cm = M.ATA(Am)
    M.ATDA_fill(Am, d, Cm)
    gp, gi, gx = Cm.csr()
    assert np.array_equal(gp, wp) and np.array_equal(gi, wi)
    dense_abs = np.zeros((n, n))
    for rows, cols, _, Ca in orc.blocks_ata(blocks, d, n):
        dense_abs[np.ix_(rows, cols)] = Ca
    rr = np.repeat(np.arange(n), np.diff(wp))
    _close(gx, wx, dense_abs[rr, wi], "ATDA stacked_pd")
    # refill: new block values and d
    X2 = [rng.standard_normal(X.shape) for X, _, _ in blocks]
    d2 = rng.uniform(0.1, 10, m)
    Am.set_values(np.concatenate([x.ravel() for x in X2]))
    M.ATDA_fill(Am, d2, Cm)
    blocks2 = [(x, rp, cp) for x, (_, rp, cp) in zip(X2, blocks)]
    Ar2 = build_ref(blocks2)
    Cr2 = ref.ATA_matrices_alloc(Ar2)
    ref.ATDA_matrices_fill_values(Ar2, d2.ctypes.data, Cr2)
    wx2 = _ref_csr(ref, Cr2)[2]
    dense_abs[:] = 0
    for rows, cols, _, Ca in orc.blocks_ata(blocks2, d2, n):
        dense_abs[np.ix_(rows, cols)] = Ca
    _close(Cm.csr()[2], wx2, dense_abs[rr, wi], "ATDA stacked_pd refill")
    for h in (Cr, Ar, Cr2, Ar2):
        ref.free_matrix(h)


def test_ATDA_permuted_dense_matches_upstream_library(sdl, orc):
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    ref = orc.reference()
    rng = np.random.default_rng(96)
    m, n = 90, 50
    rp = np.sort(rng.choice(m, 37, replace=False)).astype(np.int32)
    cp = np.sort(rng.choice(n, 29, replace=False)).astype(np.int32)
    X = rng.standard_normal((37, 29))
    d = rng.uniform(0.1, 10, m)
    Ar = ref.new_permuted_dense(m, n, 37, 29, rp.ctypes.data, cp.ctypes.data, X.ctypes.data)
    Cr = ref.ATA_matrices_alloc(Ar)
    ref.ATDA_matrices_fill_values(Ar, d.ctypes.data, Cr)
    wp, wi, wx = _ref_csr(ref, Cr)[:3]
    Am = M.permuted_dense(m, n, rp, cp, X)
    Cm = M.ATA(Am)
    M.ATDA_fill(Am, d, Cm)
    gp, gi, gx = Cm.csr()
    assert np.array_equal(gp, wp) and np.array_equal(gi, wi)
    W = X * d[rp][:, None]
    scale = (np.abs(X).T @ np.abs(W)).ravel()
    _close(gx, wx, scale, "ATDA permuted_dense")
    ref.free_matrix(Cr)
    ref.free_matrix(Ar)


# ---------------------------------------------------------------- B^T diag(d) A, B sparse, A dense blocks
@pytest.mark.parametrize("kind", ["pd", "spd"])
@pytest.mark.parametrize("use_d", [True, False])
def test_BTDA_sparse_dense_matches_upstream_library(sdl, orc, kind, use_d):
    """BTA_matrices_alloc / BTDA_matrices_fill_values (BTA without d) with B sparse and
    A permuted_dense or stacked_pd, through the drop-in C ABI, against the upstream
    library: identical structure (the columns of B that reach each block, coalesced
    as upstream's stacked_pd) and bit-identical values; then a refill."""
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    ref = orc.reference()
    rng = np.random.default_rng(97 + (kind == "spd") + 2 * use_d)
    m, n, nB = 220, 40, 150
    B = wl.small_random_csr(m, nB, 0.04, rng)
    if kind == "pd":
        blocks = [(rng.standard_normal((60, 25)), np.sort(rng.choice(m, 60, replace=False)).astype(np.int32),
                   np.sort(rng.choice(n, 25, replace=False)).astype(np.int32))]
    else:
        blocks = _spd_blocks(rng, m, n, [(30, 12), (50, 40), (7, 5), (45, 22)])
    d = rng.uniform(0.1, 10, m)

    def ref_sparse(csr):
        p, i, x, mm, nn = csr
        c = ref.new_CSR_matrix(mm, nn, len(i))
        st = c.contents
        np.ctypeslib.as_array(st.p, shape=(mm + 1,))[:] = p
        np.ctypeslib.as_array(st.i, shape=(max(1, len(i)),))[:len(i)] = i
        np.ctypeslib.as_array(st.x, shape=(max(1, len(i)),))[:len(i)] = x
        return ref.new_sparse_matrix(c)

    def ref_dense(blks):
        hs = []
        for X, rp, cp in blks:
            Xc = np.ascontiguousarray(X)
            hs.append(ref.new_permuted_dense(m, n, len(rp), len(cp), rp.ctypes.data, cp.ctypes.data, Xc.ctypes.data))
        if kind == "pd":
            return hs[0]
        arr = (C.c_void_p * len(hs))(*[C.cast(h, C.c_void_p) for h in hs])
        return ref.new_stacked_pd(m, n, len(hs), arr, None, None)

    def mine(blks):
        pds = [M.permuted_dense(m, n, rp, cp, X) for X, rp, cp in blks]
        return pds[0] if kind == "pd" else M.stacked_pd(m, n, pds)

    Br, Ar = ref_sparse(B), ref_dense(blocks)
    Cr = ref.BTA_matrices_alloc(Ar, Br)
    dd = np.ascontiguousarray(d)
    def fill_ref(A_, dv, B_, C_):
        if use_d:
            ref.BTDA_matrices_fill_values(A_, dv.ctypes.data, B_, C_)
        else:
            ref.BTA_matrices_fill_values(A_, B_, C_)

    def fill_mine(A_, dv, B_, C_):
        if use_d:
            M.BTDA_fill(A_, dv, B_, C_)
        else:
            M.mlib().BTA_matrices_fill_values(A_.ptr, B_.ptr, C_.ptr)

    fill_ref(Ar, dd, Br, Cr)
    want = _ref_csr(ref, Cr)[:3]
    Bm, Am = M.SparseMatrix.from_csr(*B), mine(blocks)
    Cm = M.BTA(Am, Bm)
    fill_mine(Am, d, Bm, Cm)
    got = Cm.csr()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    assert np.array_equal(bits(got[2]), bits(want[2]))
    # refill with new values of A, B and d
    X2 = [rng.standard_normal(X.shape) for X, _, _ in blocks]
    bx = rng.standard_normal(len(B[1]))
    d2 = rng.uniform(0.1, 10, m)
    Am.set_values(np.concatenate([x.ravel() for x in X2]))
    Bm.set_values(bx)
    fill_mine(Am, d2, Bm, Cm)
    Br2 = ref_sparse((B[0], B[1], bx, B[3], B[4]))
    Ar2 = ref_dense([(x, rp, cp) for x, (_, rp, cp) in zip(X2, blocks)])
    Cr2 = ref.BTA_matrices_alloc(Ar2, Br2)
    fill_ref(Ar2, np.ascontiguousarray(d2), Br2, Cr2)
    want2 = _ref_csr(ref, Cr2)[:3]
    assert np.array_equal(bits(Cm.csr()[2]), bits(want2[2]))
    for h in (Cr, Ar, Br, Cr2, Ar2, Br2):
        ref.free_matrix(h)
