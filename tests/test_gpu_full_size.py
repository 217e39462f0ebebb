"""Parity at the benchmark configurations' full sizes, against the CPU oracle.

Each test runs one configuration at the size it is benchmarked at, on the GPU
through the library, and compares the whole output with the oracle: structure
(row offsets and column indices) identical, values bit-identical (compared as
int64 bit patterns; the tolerance the path allows is 1e-12 relative and the
measured error is 0). The oracle runs on all host cores (``oracle.parallel``:
row ranges and independent products on a thread pool, each piece bit-identical
to the one-call result).

* 3   batched refill: all 512 B^T D A instances (rows log-uniform in 1k..64k),
      through the batch engine, every product against the oracle;
* 4a  stacked_pd (64 blocks of 64 x 256, rows permuted) x CSC 256 x 100000 with 6
      entries per column (upstream BA_spd_csr_* ->
      src/permuted_dense/permuted_dense_linalg.c:313-430);
* 4b  CSR -> CSC of a 1M x 1M matrix with 10 entries per row
      (src/sparse/CSC_matrix.c:62-123);
* 4c  coalescing of 50M COO triplets (35M distinct pairs + 15M repeats) over
      1M x 1M (oracle: upstream row_reduce, src/sparse/sparse_matrix.c:136-240);
* 5   skewed SpGEMM, A and B 1M x 1M with Zipf(1.5) row lengths (~20M nnz each,
      rows capped at 50k; src/sparse/gustavson.c:26-143).
(The 100000 x 50000 B^T D A configuration at full size is in test_gpu_device.py.)
"""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 1e-12


def _host(t, n=None):
    a = t.cpu().numpy()
    return a if n is None else a[:n]


def _assert_parity(res, what):
    assert res["structure_equal"], f"{what}: structure differs from the oracle"
    assert res["max_rel_err"] is not None and res["max_rel_err"] <= TOL, f"{what}: {res}"
    assert res["bit_identical"], f"{what}: values differ in their bits: {res}"


def _free():
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()


def test_csr_to_csc_1M_full_size(sdl, orc):
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Transpose
    A = wl.transpose_big(seed=4)
    m, n, nnz = A[3], A[4], len(A[1])
    T = Transpose(torch.as_tensor(A[0], device="cuda"), torch.as_tensor(A[1], device="cuda"), m, n)
    Tx = torch.empty(nnz, dtype=torch.float64, device="cuda")
    T.fill(torch.as_tensor(A[2], device="cuda"), Tx)
    torch.cuda.synchronize()
    want = orc.transpose(A[0], A[1], A[2], m, n)
    res = parallel.compare_csr((_host(T.Tp), _host(T.Ti), _host(Tx)), want)
    _assert_parity(res, "CSR -> CSC 1M x 1M")
    del T, Tx
    _free()


def test_coalesce_50M_full_size(sdl, orc):
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Coalesce
    rows, cols, x, m, n = wl.coalesce_device(seed=5)
    assert rows.numel() == 50_000_000
    CO = Coalesce(rows, cols, m, n)
    Cx = torch.empty(max(1, CO.nnz), dtype=torch.float64, device="cuda")
    CO.fill(x, Cx)
    # a second refill with new values (the plan is reused), some of them -0.0
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    x2 = torch.randn(x.numel(), dtype=torch.float64, device="cuda", generator=g)
    x2[::13] = -0.0
    Cx2 = torch.empty_like(Cx)
    CO.fill(x2, Cx2)
    torch.cuda.synchronize()
    hr, hc = _host(rows), _host(cols)
    got_p, got_i = _host(CO.Cp), _host(CO.Ci)
    assert CO.nnz == 35_000_000
    for xv, cx in ((x, Cx), (x2, Cx2)):
        want = parallel.coalesce(hr, hc, _host(xv), m, n)
        res = parallel.compare_csr((got_p, got_i, _host(cx, CO.nnz)), want)
        _assert_parity(res, "coalescing 50M")
    del CO, Cx, Cx2, rows, cols, x, x2
    _free()


def test_skewed_spgemm_1M_full_size(sdl, orc):
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Product
    (Ap, Ai, Ax), (Bp, Bi, Bx), _ = wl.skewed_device(seed=0)
    m = Ap.numel() - 1
    P = Product(Ap, Ai, Bp, Bi, m)
    Cx = torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda")
    P.fill(Ax, None, Bx, Cx)
    torch.cuda.synchronize()
    A = (_host(Ap), _host(Ai), _host(Ax), m, m)
    B = (_host(Bp), _host(Bi), _host(Bx), m, m)
    want = parallel.spgemm(A, B)
    res = parallel.compare_csr((_host(P.Cp), _host(P.Ci), _host(Cx, P.nnz)), want)
    _assert_parity(res, "skewed SpGEMM 1M x 1M")
    del P, Cx
    _free()


def test_batched_512_full_size(sdl, orc):
    """All 512 instances refilled by the batch engine (grouped launches replayed from
    its CUDA graph), each product compared with the oracle."""
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Batch, btda_product
    inst = wl.batched_device(seed=3, count=512)
    prods, outs = [], []
    for k in inst:
        P, T = btda_product(k["Ap"], k["Ai"], k["n"], k["Bp"], k["Bi"], k["n"])
        prods.append(P)
        outs.append(torch.empty(max(1, P.nnz), dtype=torch.float64, device="cuda"))
    Bt = Batch(prods)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    s = torch.cuda.Stream()
    for rnd in range(2):  # eager first refill, then a graph replay with new values
        for i, k in enumerate(inst):
            k["Ax"] = torch.randn(k["Ai"].numel(), generator=g, device="cuda", dtype=torch.float64)
            k["Bx"] = torch.randn(k["Bi"].numel(), generator=g, device="cuda", dtype=torch.float64)
            k["d"] = torch.rand(k["m"], generator=g, device="cuda", dtype=torch.float64) * 9.9 + 0.1
            Bt.bind(i, k["Bx"], k["d"], k["Ax"], outs[i])
        with torch.cuda.stream(s):
            Bt.refill(stream=s)
        s.synchronize()

    def one(i):
        k, P = inst[i], prods[i]
        got = (_host(P.Cp), _host(P.Ci), _host(outs[i], P.nnz))
        want = orc.btda((_host(k["Ap"]), _host(k["Ai"]), _host(k["Ax"]), k["m"], k["n"]),
                        (_host(k["Bp"]), _host(k["Bi"]), _host(k["Bx"]), k["m"], k["n"]), _host(k["d"]))
        return parallel.compare_csr(got, want)

    results = parallel.map_threads(one, range(len(inst)))
    bad = [i for i, r in enumerate(results) if not (r["structure_equal"] and r["bit_identical"])]
    assert not bad, f"products differing from the oracle: {bad[:10]}"
    assert max(r["max_rel_err"] for r in results) == 0.0
    del Bt, prods, outs
    _free()


def test_stacked_pd_x_csc_full_size(sdl, orc):
    """64 blocks of 64 x 256 (rows a random permutation of 4096) times S 256 x 100000
    with 6 distinct rows per column: 64 output blocks of 64 x 100000."""
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import BlocksCsr
    rng = np.random.default_rng(6)
    nb, m0, n0, S_n = 64, 64, 256, 100_000
    X = rng.standard_normal((nb, m0, n0))
    cperm = np.arange(n0, dtype=np.int32)
    St = wl.fixed_rowlen_csr(S_n, n0, 6, rng)
    Sp, Si, Sx = orc.transpose(St[0], St[1], St[2], S_n, n0)
    P = BlocksCsr([m0] * nb, [n0] * nb, [cperm] * nb, Sp, Si, n0, S_n)
    Cv = torch.empty(P.c_values, dtype=torch.float64, device="cuda")
    P.fill(torch.as_tensor(X.ravel(), device="cuda"), torch.as_tensor(Sx, device="cuda"), Cv)
    torch.cuda.synchronize()
    got = Cv.cpu().numpy()
    assert P.out_blocks == nb
    offs = np.concatenate([[0], np.cumsum([b[1] * b[2] for b in P.blocks])])

    def one(k):
        src, mk, n0c, perm = P.blocks[k]
        (cols, Cw), = orc.blocks_csr([(X[src], cperm)], Sp, Si, Sx, S_n)
        Cg = got[offs[k]:offs[k + 1]].reshape(mk, n0c)
        return (src == k and np.array_equal(perm, cols) and
                np.array_equal(Cg.view(np.int64), Cw.view(np.int64)))

    ok = parallel.map_threads(one, range(P.out_blocks))
    assert all(ok), f"blocks differing from the oracle: {[k for k, v in enumerate(ok) if not v][:10]}"
    del P, Cv
    _free()
