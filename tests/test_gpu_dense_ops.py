"""Every permuted_dense / stacked_pd operation of the drop-in C ABI that runs a
dense-block fill program, against the same calls on the upstream library compiled
from its sources: B^T diag(d) A and B^T A with a dense-block B, B A with a
dense-block A, DA, transpose, row_gather and row_reduce.

The structure must be identical: the CSR view, and for a stacked_pd its blocks
(row and column perms) and its source-block map. Values must be bit-identical
where upstream's arithmetic is scalar (copies, scalings, sparse x dense sums), and
within 1e-12 of the sum of |terms| of each cell where upstream calls cblas_dgemm
(dense x dense products), whose summation order is unspecified. Every case is
filled twice: once at alloc values, once after new values of every operand."""
import ctypes as C

import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl
from sparsediff_linalg_b200._lib import CSR_p, matrix, matrix_p

pytestmark = pytest.mark.gpu

PD, SPD = 1, 2
c_int_p = C.POINTER(C.c_int)


class _PD(C.Structure):
    """Leading fields of a permuted_dense (the same in both libraries)."""
    _fields_ = [("base", matrix), ("m0", C.c_int), ("n0", C.c_int), ("row_perm", c_int_p),
                ("col_perm", c_int_p)]


class _SPD(C.Structure):
    _fields_ = [("base", matrix), ("n_blocks", C.c_int), ("blocks", C.POINTER(C.POINTER(_PD))),
                ("src_p", c_int_p), ("src_i", c_int_p)]


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


# ----------------------------------------------------------------- operands
def pd_spec(rng, m, n, m0, n0):
    rp = np.sort(rng.choice(m, m0, replace=False)).astype(np.int32)
    cp = np.sort(rng.choice(n, n0, replace=False)).astype(np.int32)
    return ("pd", m, n, [(rng.standard_normal((m0, n0)), rp, cp)])


def spd_spec(rng, m, n, shapes, rows=None):
    """Row-disjoint blocks with overlapping column sets; `rows` the pool of rows."""
    pool = rng.permutation(m if rows is None else rows)
    blocks, at = [], 0
    for m0, n0 in shapes:
        rp = np.sort(pool[at:at + m0]).astype(np.int32)
        at += m0
        cp = np.sort(rng.choice(n, n0, replace=False)).astype(np.int32)
        blocks.append((rng.standard_normal((m0, n0)), rp, cp))
    return ("spd", m, n, blocks)


def sparse_spec(rng, m, n, density):
    return ("sparse", wl.small_random_csr(m, n, density, rng))


def dense_of(spec):
    if spec[0] == "sparse":
        p, i, x, m, n = spec[1]
        D = np.zeros((m, n))
        for r in range(m):
            D[r, i[p[r]:p[r + 1]]] = x[p[r]:p[r + 1]]
        return D
    _, m, n, blocks = spec
    D = np.zeros((m, n))
    for X, rp, cp in blocks:
        D[np.ix_(rp, cp)] = X
    return D


def values_of(spec):
    if spec[0] == "sparse":
        return np.asarray(spec[1][2], np.float64)
    return np.concatenate([X.ravel() for X, _, _ in spec[3]] + [np.zeros(0)])


def renewed(spec, rng):
    """The same structure with new values."""
    if spec[0] == "sparse":
        p, i, x, m, n = spec[1]
        return ("sparse", (p, i, rng.standard_normal(len(x)), m, n))
    return (spec[0], spec[1], spec[2], [(rng.standard_normal(X.shape), rp, cp) for X, rp, cp in spec[3]])


class Lib:
    """One library (the upstream one or this one) behind the same C ABI."""

    def __init__(self, L):
        self.L = L

    def make(self, spec):
        L = self.L
        if spec[0] == "sparse":
            p, i, x, m, n = spec[1]
            c = L.new_CSR_matrix(m, n, len(i))
            s = c.contents
            np.ctypeslib.as_array(s.p, shape=(m + 1,))[:] = p
            if len(i):
                np.ctypeslib.as_array(s.i, shape=(len(i),))[:] = i
                np.ctypeslib.as_array(s.x, shape=(len(i),))[:] = x
            return L.new_sparse_matrix(c)
        kind, m, n, blocks = spec
        hs = []
        for X, rp, cp in blocks:
            Xc = np.ascontiguousarray(X)
            hs.append(L.new_permuted_dense(m, n, len(rp), len(cp), rp.ctypes.data, cp.ctypes.data, Xc.ctypes.data))
        if kind == "pd":
            return hs[0]
        arr = (C.c_void_p * max(1, len(hs)))(*[C.cast(h, C.c_void_p) for h in hs])
        return L.new_stacked_pd(m, n, len(hs), arr, None, None)

    @staticmethod
    def set_values(h, x):
        """Overwrite a handle's values (all kinds keep them at base.x) and bump its version."""
        x = np.asarray(x, np.float64)
        if len(x):
            np.ctypeslib.as_array(h.contents.x, shape=(len(x),))[:] = x
        h.contents.values_version += 1

    def free(self, *hs):
        for h in hs:
            self.L.free_matrix(h)


def csr_of(h):
    from sparsediff_linalg_b200.host import csr_from_ptr
    return csr_from_ptr(C.CFUNCTYPE(CSR_p, matrix_p)(h.contents.to_csr)(h))[:3]


def structure_of(h):
    """Blocks (row perm, col perm) and the source map of a dense-block handle
    (nothing for a sparse one)."""
    kind = h.contents.kind
    if kind == 0:
        return [], None
    if kind == PD:
        p = C.cast(h, C.POINTER(_PD)).contents
        return [(np.ctypeslib.as_array(p.row_perm, shape=(p.m0,)).copy() if p.m0 else np.zeros(0, np.int32),
                 np.ctypeslib.as_array(p.col_perm, shape=(p.n0,)).copy() if p.n0 else np.zeros(0, np.int32))], None
    assert kind == SPD
    s = C.cast(h, C.POINTER(_SPD)).contents
    blocks = []
    for k in range(s.n_blocks):
        p = s.blocks[k].contents
        blocks.append((np.ctypeslib.as_array(p.row_perm, shape=(p.m0,)).copy() if p.m0 else np.zeros(0, np.int32),
                       np.ctypeslib.as_array(p.col_perm, shape=(p.n0,)).copy() if p.n0 else np.zeros(0, np.int32)))
    sp = np.ctypeslib.as_array(s.src_p, shape=(s.n_blocks + 1,)).copy()
    si = np.ctypeslib.as_array(s.src_i, shape=(int(sp[-1]),)).copy() if sp[-1] else np.zeros(0, np.int32)
    return blocks, (sp, si)


def assert_same(got_h, want_h, exact, absbound=None, what=""):
    assert got_h.contents.kind == want_h.contents.kind, what
    assert (got_h.contents.m, got_h.contents.n, got_h.contents.nnz) == \
        (want_h.contents.m, want_h.contents.n, want_h.contents.nnz), what
    gb, gs = structure_of(got_h)
    wb, ws = structure_of(want_h)
    assert len(gb) == len(wb), what
    for (gr, gc), (wr, wc) in zip(gb, wb):
        assert np.array_equal(gr, wr) and np.array_equal(gc, wc), what
    if ws is not None:
        assert np.array_equal(gs[0], ws[0]) and np.array_equal(gs[1], ws[1]), what
    gp, gi, gx = csr_of(got_h)
    wp, wi, wx = csr_of(want_h)
    assert np.array_equal(gp, wp) and np.array_equal(gi, wi), what
    if exact:
        assert np.array_equal(bits(gx), bits(wx)), what
    else:
        rows = np.repeat(np.arange(len(wp) - 1), np.diff(wp))
        bound = 1e-12 * absbound[rows, wi] + 1e-300
        err = np.abs(gx - wx)
        assert np.all(err <= bound), f"{what}: max err/bound {np.max(err / bound)}"


@pytest.fixture(scope="module")
def libs(sdl, orc):
    if not orc.reference_available():
        pytest.skip("upstream library not built")
    from sparsediff_linalg_b200 import matrices as M
    return Lib(M.mlib()), Lib(orc.reference())


# ----------------------------------------------------------------- operand sets
def _left_dense(rng, kind, m, n):
    if kind == "pd":
        return pd_spec(rng, m, n, 70, 23)
    # one block on rows no other operand uses, one 1 x 1 block, uneven shapes
    return spd_spec(rng, m, n, [(13, 20), (25, 45), (1, 1), (30, 17), (6, 50)])


def _right(rng, kind, m, n):
    if kind == "pd":
        return pd_spec(rng, m, n, 55, 37)
    if kind == "spd":
        return spd_spec(rng, m, n, [(20, 30), (9, 7), (33, 60), (17, 16)])
    return sparse_spec(rng, m, n, 0.05)


# ----------------------------------------------------------------- B^T diag(d) A, B dense blocks
@pytest.mark.parametrize("bk", ["pd", "spd"])
@pytest.mark.parametrize("ak", ["pd", "spd", "sparse"])
@pytest.mark.parametrize("use_d", [True, False])
def test_BTDA_dense_left_matches_upstream(libs, bk, ak, use_d):
    mine, ref = libs
    rng = np.random.default_rng(300 + 7 * ["pd", "spd"].index(bk) + ["pd", "spd", "sparse"].index(ak) + 50 * use_d)
    m = 120
    Bs, As = _left_dense(rng, bk, m, 50), _right(rng, ak, m, 60)
    exact = ak == "sparse"
    for it in range(2):
        d = rng.uniform(0.1, 10, m)
        dd = np.ascontiguousarray(d)
        hs = {}
        for name, lib in (("mine", mine), ("ref", ref)):
            B, A = lib.make(Bs), lib.make(As)
            Cm = lib.L.BTA_matrices_alloc(A, B)
            if use_d:
                lib.L.BTDA_matrices_fill_values(A, dd.ctypes.data, B, Cm)
            else:
                lib.L.BTA_matrices_fill_values(A, B, Cm)
            hs[name] = (B, A, Cm)
        dabs = np.abs(d) if use_d else np.ones(m)
        absb = np.abs(dense_of(Bs)).T @ (dabs[:, None] * np.abs(dense_of(As)))
        assert_same(hs["mine"][2], hs["ref"][2], exact, absb, f"BT{'D' if use_d else ''}A {bk} x {ak} #{it}")
        if it == 0:
            # refill the same outputs after new values of every operand
            Bs2, As2 = renewed(Bs, rng), renewed(As, rng)
            d2 = np.ascontiguousarray(rng.uniform(0.1, 10, m))
            for name, lib in (("mine", mine), ("ref", ref)):
                B, A, Cm = hs[name]
                Lib.set_values(B, values_of(Bs2))
                Lib.set_values(A, values_of(As2))
                if use_d:
                    lib.L.BTDA_matrices_fill_values(A, d2.ctypes.data, B, Cm)
                else:
                    lib.L.BTA_matrices_fill_values(A, B, Cm)
            dabs = np.abs(d2) if use_d else np.ones(m)
            absb = np.abs(dense_of(Bs2)).T @ (dabs[:, None] * np.abs(dense_of(As2)))
            assert_same(hs["mine"][2], hs["ref"][2], exact, absb, f"refill {bk} x {ak}")
        for name, lib in (("mine", mine), ("ref", ref)):
            lib.free(*hs[name][::-1])


# ----------------------------------------------------------------- B A with A dense blocks
@pytest.mark.parametrize("bk,ak", [("pd", "pd"), ("pd", "spd"), ("sparse", "pd"), ("sparse", "spd")])
def test_BA_dense_right_matches_upstream(libs, bk, ak):
    mine, ref = libs
    rng = np.random.default_rng(400 + 3 * ["pd", "sparse"].index(bk) + ["pd", "spd"].index(ak))
    mB, k, n = 80, 120, 60
    Bs = pd_spec(rng, mB, k, 40, 70) if bk == "pd" else sparse_spec(rng, mB, k, 0.05)
    As = _right(rng, ak, k, n)
    exact = bk == "sparse"
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        B, A = lib.make(Bs), lib.make(As)
        Cm = lib.L.BA_matrices_alloc(B, A)
        lib.L.BA_matrices_fill_values(B, A, Cm)
        hs[name] = (B, A, Cm)
    absb = np.abs(dense_of(Bs)) @ np.abs(dense_of(As))
    assert_same(hs["mine"][2], hs["ref"][2], exact, absb, f"BA {bk} x {ak}")
    Bs2, As2 = renewed(Bs, rng), renewed(As, rng)
    for name, lib in (("mine", mine), ("ref", ref)):
        B, A, Cm = hs[name]
        Lib.set_values(B, values_of(Bs2))
        Lib.set_values(A, values_of(As2))
        lib.L.BA_matrices_fill_values(B, A, Cm)
    absb = np.abs(dense_of(Bs2)) @ np.abs(dense_of(As2))
    assert_same(hs["mine"][2], hs["ref"][2], exact, absb, f"BA refill {bk} x {ak}")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])


# ----------------------------------------------------------------- DA, transpose
def _dense_operand(rng, kind, m, n):
    if kind == "pd":
        return pd_spec(rng, m, n, 37, 29)
    return spd_spec(rng, m, n, [(11, 20), (30, 45), (1, 1), (9, 33)])


@pytest.mark.parametrize("kind", ["pd", "spd"])
def test_DA_and_transpose_match_upstream(libs, kind):
    mine, ref = libs
    rng = np.random.default_rng(500 + (kind == "spd"))
    m, n = 90, 70
    As = _dense_operand(rng, kind, m, n)
    d = np.ascontiguousarray(rng.uniform(-3, 3, m))
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        A = lib.make(As)
        D = lib.L.copy_sparsity_matrices_alloc(A)
        lib.L.DA_matrices_fill_values(d.ctypes.data, A, D)
        T = lib.L.transpose_matrices_alloc(A)
        lib.L.transpose_matrices_fill_values(A, T)
        hs[name] = (A, D, T)
    assert_same(hs["mine"][1], hs["ref"][1], True, what=f"DA {kind}")
    assert_same(hs["mine"][2], hs["ref"][2], True, what=f"transpose {kind}")
    As2 = renewed(As, rng)
    d2 = np.ascontiguousarray(rng.uniform(-3, 3, m))
    for name, lib in (("mine", mine), ("ref", ref)):
        A, D, T = hs[name]
        Lib.set_values(A, values_of(As2))
        lib.L.DA_matrices_fill_values(d2.ctypes.data, A, D)
        lib.L.transpose_matrices_fill_values(A, T)
    assert_same(hs["mine"][1], hs["ref"][1], True, what=f"DA refill {kind}")
    assert_same(hs["mine"][2], hs["ref"][2], True, what=f"transpose refill {kind}")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])


# ----------------------------------------------------------------- row_gather, row_reduce
_alloc_t = C.CFUNCTYPE(matrix_p, matrix_p, c_int_p, C.c_int)
_fill_t = C.CFUNCTYPE(None, matrix_p, matrix_p)


@pytest.mark.parametrize("kind", ["pd", "spd"])
def test_row_gather_and_row_reduce_match_upstream(libs, kind):
    mine, ref = libs
    rng = np.random.default_rng(600 + (kind == "spd"))
    m, n, m_out = 90, 70, 40
    As = _dense_operand(rng, kind, m, n)
    mp = np.ascontiguousarray(rng.integers(0, m, 130), np.int32)     # repeats, rows outside the blocks
    group = np.ascontiguousarray(rng.integers(0, m_out, m), np.int32)
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        A = lib.make(As)
        G = _alloc_t(A.contents.row_gather_alloc)(A, mp.ctypes.data_as(c_int_p), len(mp))
        _fill_t(A.contents.row_gather_fill_values)(A, G)
        R = _alloc_t(A.contents.row_reduce_alloc)(A, group.ctypes.data_as(c_int_p), m_out)
        _fill_t(A.contents.row_reduce_fill_values)(A, R)
        hs[name] = (A, G, R)
    assert_same(hs["mine"][1], hs["ref"][1], True, what=f"row_gather {kind}")
    assert_same(hs["mine"][2], hs["ref"][2], True, what=f"row_reduce {kind}")
    As2 = renewed(As, rng)
    for name, lib in (("mine", mine), ("ref", ref)):
        A, G, R = hs[name]
        Lib.set_values(A, values_of(As2))
        _fill_t(A.contents.row_gather_fill_values)(A, G)
        _fill_t(A.contents.row_reduce_fill_values)(A, R)
    assert_same(hs["mine"][1], hs["ref"][1], True, what=f"row_gather refill {kind}")
    assert_same(hs["mine"][2], hs["ref"][2], True, what=f"row_reduce refill {kind}")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])
