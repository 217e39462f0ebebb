"""Kronecker products and the dense-vector helpers through the drop-in C ABI,
against the same calls on the upstream library compiled from its sources
(upstream src/matmul_kron_dispatchers.c, src/stacked_pd/stacked_pd_kron_linalg.c,
src/support/mini_numpy.c). Structure identical; values bit-identical except where
upstream calls cblas_dgemm (a dense A against a dense-block J, and the dense
kron-vector product), compared there within 1e-12 of the sum of |terms|."""
import ctypes as C

import numpy as np
import pytest

from sparsediff_linalg_b200._lib import matrix_p

from test_gpu_dense_ops import (Lib, assert_same, dense_of, pd_spec, renewed, sparse_spec, spd_spec,
                                values_of)

pytestmark = pytest.mark.gpu

vp, ci = C.c_void_p, C.c_int
SIGS = {
    "BA_kron_vec_matrices": (None, [matrix_p, vp, vp, ci]),
    "BA_kron_matrices_alloc": (matrix_p, [matrix_p, ci, matrix_p]),
    "BA_kron_matrices_fill_values": (None, [matrix_p, ci, matrix_p, matrix_p]),
    "BA_dense_kron_I_matrices_alloc": (matrix_p, [matrix_p, ci, matrix_p]),
    "BA_dense_kron_I_matrices_fill_values": (None, [matrix_p, ci, matrix_p, matrix_p]),
    "repeat": (None, [vp, vp, ci, ci]),
    "tile_double": (None, [vp, vp, ci, ci]),
    "scaled_ones": (None, [vp, ci, C.c_double]),
    "A_transpose": (None, [vp, vp, ci, ci]),
    "Y_kron_I_vec": (None, [ci, ci, ci, vp, vp, vp]),
    "I_kron_XT_vec": (None, [ci, ci, ci, vp, vp, vp]),
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


def full_pd(rng, m, n):
    return ("pd", m, n, [(rng.standard_normal((m, n)), np.arange(m, dtype=np.int32),
                          np.arange(n, dtype=np.int32))])


def _J(rng, kind, rows, n):
    if kind == "pd":
        return pd_spec(rng, rows, n, rows // 2, 13)
    if kind == "spd":
        return spd_spec(rng, rows, n, [(3, 9), (4, 20), (1, 1)])
    return sparse_spec(rng, rows, n, 0.2)


@pytest.mark.parametrize("akind", ["pd", "sparse"])
@pytest.mark.parametrize("jkind", ["pd", "spd", "sparse"])
@pytest.mark.parametrize("layout", ["I_A", "A_I"])
def test_kron_products_match_upstream(libs, akind, jkind, layout):
    if akind == "sparse" and layout == "A_I":
        pytest.skip("kron(A, I) is defined for a full permuted_dense A only")
    mine, ref = libs
    rng = np.random.default_rng(800 + 10 * ["pd", "sparse"].index(akind) + ["pd", "spd", "sparse"].index(jkind)
                                + 100 * (layout == "A_I"))
    m, n, p, nJ = 4, 5, 3, 24
    As = full_pd(rng, m, n) if akind == "pd" else sparse_spec(rng, m, n, 0.5)
    Js = _J(rng, jkind, p * n, nJ)
    exact = akind == "sparse" or jkind == "sparse"
    alloc = "BA_kron_matrices_alloc" if layout == "I_A" else "BA_dense_kron_I_matrices_alloc"
    fill = "BA_kron_matrices_fill_values" if layout == "I_A" else "BA_dense_kron_I_matrices_fill_values"

    def kron_dense(a_spec, j_spec):
        Ad = np.abs(dense_of(a_spec))
        K = np.kron(np.eye(p), Ad) if layout == "I_A" else np.kron(Ad, np.eye(p))
        return K @ np.abs(dense_of(j_spec))

    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        A, J = lib.make(As), lib.make(Js)
        Cm = getattr(lib.L, alloc)(A, p, J)
        getattr(lib.L, fill)(A, p, J, Cm)
        hs[name] = (A, J, Cm)
    assert_same(hs["mine"][2], hs["ref"][2], exact, kron_dense(As, Js), f"kron {akind} x {jkind} {layout}")
    As2, Js2 = renewed(As, rng), renewed(Js, rng)
    for name, lib in (("mine", mine), ("ref", ref)):
        A, J, Cm = hs[name]
        Lib.set_values(A, values_of(As2))
        Lib.set_values(J, values_of(Js2))
        getattr(lib.L, fill)(A, p, J, Cm)
    assert_same(hs["mine"][2], hs["ref"][2], exact, kron_dense(As2, Js2), f"kron refill {akind} x {jkind}")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])


def test_kron_p1_is_BA(libs):
    mine, ref = libs
    rng = np.random.default_rng(820)
    As, Js = sparse_spec(rng, 6, 9, 0.4), spd_spec(rng, 9, 11, [(3, 4), (5, 7)])
    hs = {}
    for name, lib in (("mine", mine), ("ref", ref)):
        A, J = lib.make(As), lib.make(Js)
        Cm = lib.L.BA_kron_matrices_alloc(A, 1, J)
        lib.L.BA_kron_matrices_fill_values(A, 1, J, Cm)
        hs[name] = (A, J, Cm)
    assert_same(hs["mine"][2], hs["ref"][2], True, None, "kron p=1")
    for name, lib in (("mine", mine), ("ref", ref)):
        lib.free(*hs[name][::-1])


@pytest.mark.parametrize("akind", ["pd", "sparse"])
def test_kron_vec_matches_upstream(libs, akind):
    mine, ref = libs
    rng = np.random.default_rng(830 + (akind == "sparse"))
    m, n, p = 37, 29, 5
    As = full_pd(rng, m, n) if akind == "pd" else sparse_spec(rng, m, n, 0.3)
    x = np.ascontiguousarray(rng.standard_normal(p * n))
    ys = []
    for lib in (mine, ref):
        A = lib.make(As)
        y = np.zeros(p * m)
        lib.L.BA_kron_vec_matrices(A, x.ctypes.data, y.ctypes.data, p)
        ys.append(y)
        lib.free(A)
    if akind == "sparse":
        assert np.array_equal(bits(ys[0]), bits(ys[1]))
    else:
        bound = 1e-12 * (np.abs(x.reshape(p, n)) @ np.abs(dense_of(As)).T).ravel() + 1e-300
        assert np.all(np.abs(ys[0] - ys[1]) <= bound)


def test_dense_helpers_match_upstream(libs):
    mine, ref = libs
    rng = np.random.default_rng(840)
    a = np.ascontiguousarray(rng.standard_normal(23))
    m, k, n = 7, 5, 9
    Y = np.ascontiguousarray(rng.standard_normal(k * n))
    X = np.ascontiguousarray(rng.standard_normal(m * k))
    w = np.ascontiguousarray(rng.standard_normal(m * n))
    A = np.ascontiguousarray(rng.standard_normal((13, 17)))
    outs = []
    for lib in (mine, ref):
        L = lib.L
        r = {}
        r["repeat"] = np.zeros(23 * 4)
        L.repeat(r["repeat"].ctypes.data, a.ctypes.data, 23, 4)
        r["tile"] = np.zeros(23 * 3)
        L.tile_double(r["tile"].ctypes.data, a.ctypes.data, 23, 3)
        r["ones"] = np.zeros(11)
        L.scaled_ones(r["ones"].ctypes.data, 11, -2.5)
        r["AT"] = np.zeros(13 * 17)
        L.A_transpose(r["AT"].ctypes.data, A.ctypes.data, 13, 17)
        r["ykron"] = np.zeros(m * k)
        L.Y_kron_I_vec(m, k, n, Y.ctypes.data, w.ctypes.data, r["ykron"].ctypes.data)
        r["ikron"] = np.zeros(k * n)
        L.I_kron_XT_vec(m, k, n, X.ctypes.data, w.ctypes.data, r["ikron"].ctypes.data)
        outs.append(r)
    for key in outs[0]:
        assert np.array_equal(bits(outs[0][key]), bits(outs[1][key])), key
