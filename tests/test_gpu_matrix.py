"""GPU parity of the upstream polymorphic matrix API (sparse kind): dispatchers
BTA/BTDA/BA/ATA/ATDA/DA/transpose and the row_gather / row_reduce vtable slots,
against the CPU oracle bit for bit, plus the version/cache protocol (upstream
tests/test_cache_coherence.h): fills refresh operand mirrors iff values_version
moved and bump the output's version."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


def same(got, want):
    gp, gi, gx = got
    wp, wi, wx = want[:3]
    assert np.array_equal(gp, wp) and np.array_equal(gi, wi)
    assert np.array_equal(bits(gx), bits(wx))


@pytest.fixture
def M(sdl):
    from sparsediff_linalg_b200 import matrices
    return matrices


def test_btda_dispatch_and_cache_coherence(M, orc):
    rng = np.random.default_rng(31)
    A = wl.small_random_csr(400, 300, 0.02, rng)
    B = wl.small_random_csr(400, 200, 0.02, rng)
    Am = M.SparseMatrix.from_csr(*A)
    Bm = M.SparseMatrix.from_csr(*B)
    C = M.BTA(Am, Bm)
    assert C.kind == 0
    d = rng.uniform(0.1, 10, 400)
    v0 = C.version
    M.BTDA_fill(Am, d, Bm, C)
    assert C.version == v0 + 1
    same(C.csr(), orc.btda(A, B, d))
    # change B's values only: the fill must see them (stale mirror otherwise)
    bx = rng.standard_normal(len(B[1]))
    Bm.set_values(bx)
    M.BTDA_fill(Am, d, Bm, C)
    same(C.csr(), orc.btda(A, (B[0], B[1], bx, B[3], B[4]), d))
    # BTA (d = NULL)
    C.BTDA_fill(Am, None, Bm)
    same(C.csr(), orc.btda(A, (B[0], B[1], bx, B[3], B[4]), None))


def test_ba_and_chained_products(M, orc):
    """C = B A, then E = C^T D C reading C's device values without re-upload."""
    rng = np.random.default_rng(32)
    Bx = wl.small_random_csr(150, 120, 0.05, rng)
    Ax = wl.small_random_csr(120, 90, 0.05, rng)
    Bm = M.SparseMatrix.from_csr(*Bx)
    Am = M.SparseMatrix.from_csr(*Ax)
    Cm = M.BA(Bm, Am)
    M.BA_fill(Bm, Am, Cm)
    want = orc.spgemm(Bx, Ax)
    same(Cm.csr(), want)
    Em = M.ATA(Cm)
    d = rng.uniform(0.1, 10, 150)
    M.ATDA_fill(Cm, d, Em)
    Cc = (want[0], want[1], want[2], 150, 90)
    same(Em.csr(), orc.btda(Cc, Cc, d))


def test_transpose_da_copy_sparsity(M, orc):
    rng = np.random.default_rng(33)
    A = wl.small_random_csr(200, 170, 0.05, rng)
    Am = M.SparseMatrix.from_csr(*A)
    AT = M.transpose(Am)
    M.transpose_fill(Am, AT)
    same(AT.csr(), orc.transpose(A[0], A[1], A[2], 200, 170))
    Dm = M.copy_sparsity(Am)
    d = rng.uniform(-2, 2, 200)
    M.DA_fill(d, Am, Dm)
    rows = np.repeat(np.arange(200), np.diff(A[0]))
    same(Dm.csr(), (A[0], A[1], A[2] * d[rows]))


def test_row_gather_and_reduce(M, orc):
    rng = np.random.default_rng(34)
    A = wl.small_random_csr(300, 80, 0.05, rng)
    Am = M.SparseMatrix.from_csr(*A)
    mp = rng.integers(0, 300, 500)           # repeats allowed (cvxpy#3442)
    G = Am.row_gather(mp)
    Am.row_gather_fill(G)
    same(G.csr(), orc.row_gather(A[0], A[1], A[2], mp))
    group = rng.integers(0, 40, 300)
    R = Am.row_reduce(group, 40)
    Am.row_reduce_fill(R)
    same(R.csr(), orc.row_reduce(A[0], A[1], A[2], 300, 80, group, 40))
    x2 = rng.standard_normal(len(A[1]))
    Am.set_values(x2)
    Am.row_reduce_fill(R)
    same(R.csr(), orc.row_reduce(A[0], A[1], x2, 300, 80, group, 40))


def test_matrix_api_matches_upstream_library(M, orc):
    """Same call sequence through the upstream library itself (compiled from its
    sources) -- when it is available on this machine."""
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    import ctypes as C
    from sparsediff_linalg_b200.host import csr_from_ptr
    ref = orc.reference()
    rng = np.random.default_rng(35)
    A = wl.small_random_csr(500, 300, 0.02, rng)
    B = wl.small_random_csr(500, 250, 0.02, rng)
    d = rng.uniform(0.1, 10, 500)

    def ref_mat(csr):
        p, i, x, m, n = csr
        c = ref.new_CSR_matrix(m, n, len(i))
        s = c.contents
        np.ctypeslib.as_array(s.p, shape=(m + 1,))[:] = p
        np.ctypeslib.as_array(s.i, shape=(len(i),))[:] = i
        np.ctypeslib.as_array(s.x, shape=(len(i),))[:] = x
        return ref.new_sparse_matrix(c)

    Ar, Br = ref_mat(A), ref_mat(B)
    Cr = ref.BTA_matrices_alloc(Ar, Br)
    dd = np.ascontiguousarray(d)
    ref.BTDA_matrices_fill_values(Ar, dd.ctypes.data, Br, Cr)
    to_csr = C.CFUNCTYPE(C.POINTER(__import__("sparsediff_linalg_b200._lib", fromlist=["x"]).CSR_matrix),
                         C.POINTER(__import__("sparsediff_linalg_b200._lib", fromlist=["x"]).matrix))
    rp, ri, rx, _, _ = csr_from_ptr(to_csr(Cr.contents.to_csr)(Cr))
    Am = M.SparseMatrix.from_csr(*A)
    Bm = M.SparseMatrix.from_csr(*B)
    Cm = M.BTA(Am, Bm)
    M.BTDA_fill(Am, d, Bm, Cm)
    same(Cm.csr(), (rp, ri, rx))
    ref.free_matrix(Cr)
    ref.free_matrix(Ar)
    ref.free_matrix(Br)
