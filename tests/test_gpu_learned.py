"""Learned row scheduler: the CUDA training kernels' gradients against the FP64 CPU
oracle, training, exactness of the learned symbolic pass (it may only change the
schedule, never the product) and what the trained network gains."""
import numpy as np
import pytest

from sparsediff_linalg_b200 import workloads as wl
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _skewed(seed, m=20000, target=400_000, cap=2000):
    (Ap, Ai, Ax), (Bp, Bi, Bx), _ = wl.skewed_device(seed=seed, m=m, n=m, target=target, cap=cap)
    return (Ap, Ai, Ax), (Bp, Bi, Bx)


def _spgemm(A, B, n):
    from sparsediff_linalg_b200.device import Product
    return Product(A[0], A[1], B[0], B[1], n)


def test_gradients_match_cpu_oracle(sdl):
    import torch
    from sparsediff_linalg_b200.learned import Mlp, row_stats
    A, B = _skewed(1)
    P = _spgemm(A, B, 20000)
    feat, label = row_stats(P)
    idx = torch.randperm(feat.shape[0], generator=torch.Generator().manual_seed(0))[:700].cuda()
    f, l = feat[idx].contiguous(), label[idx].contiguous()
    net = Mlp(seed=3)
    rng = np.random.default_rng(3)
    net.set_params((rng.standard_normal(mo.NPARAMS) * 0.2).astype(np.float32))
    loss, g = net.gradient(f, l)
    lc, gc = mo.loss_and_grad(net.params().astype(np.float64), f.cpu().numpy().astype(np.float64),
                              l.cpu().numpy().astype(np.float64))
    # FP32 kernels vs the FP64 oracle
    assert abs(loss - lc) <= 1e-4 * max(1.0, abs(lc))
    assert np.max(np.abs(g - gc)) <= 1e-4 * max(1.0, np.max(np.abs(gc))), np.max(np.abs(g - gc))


def _train(sdl, seeds=(10, 11, 12, 13), epochs=12):
    import torch
    from sparsediff_linalg_b200.learned import Mlp, row_stats
    feats, labels = [], []
    for sd in seeds:
        A, B = _skewed(sd)
        P = _spgemm(A, B, 20000)
        f, l = row_stats(P)
        feats.append(f)
        labels.append(l)
    F, L = torch.cat(feats), torch.cat(labels)
    net = Mlp(seed=7)
    first, _ = net.gradient(F, L)
    last = net.train(F, L, epochs=epochs, batch=4096, lr=3e-3, seed=1)
    return net, first, last


def test_training_reduces_loss(sdl):
    net, first, last = _train(sdl)
    assert last < 0.5 * first, (first, last)


@pytest.mark.parametrize("mode", ["untrained", "trained", "zero_margin"])
def test_learned_product_is_exactly_the_product(sdl, mode):
    import torch
    from sparsediff_linalg_b200.device import Product
    from sparsediff_linalg_b200.learned import LearnedProduct, Mlp
    if mode == "untrained":
        net, margin = Mlp(seed=5), 0.25
    else:
        net, _, _ = _train(sdl, seeds=(20, 21), epochs=6)
        margin = 0.25 if mode == "trained" else 0.0
    A, B = _skewed(99)
    P = Product(A[0], A[1], B[0], B[1], 20000)
    Q = LearnedProduct(A[0], A[1], B[0], B[1], 20000, net, margin=margin)
    assert P.nnz == Q.nnz
    assert torch.equal(P.Cp, Q.Cp) and torch.equal(P.Ci, Q.Ci)
    cp = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    cq = torch.empty(Q.nnz, dtype=torch.float64, device="cuda")
    P.fill(A[2], None, B[2], cp)
    Q.fill(A[2], None, B[2], cq)
    torch.cuda.synchronize()
    assert torch.equal(cp.view(torch.int64), cq.view(torch.int64))
    if mode == "untrained":
        assert Q.stats["fallback_rows"] > 0  # the exact pass did step in


def test_trained_network_gain(sdl):
    """On a held-out matrix the trained network sizes the column scratch close to
    the true output (well below the term-count bound the plain pass reserves),
    with few rows falling back to the exact pass, and predicts most classes."""
    from sparsediff_linalg_b200.device import Product
    from sparsediff_linalg_b200.learned import LearnedProduct, scratch_bytes
    net, _, _ = _train(sdl)
    A, B = _skewed(123)
    plain = Product(A[0], A[1], B[0], B[1], 20000)
    learned = LearnedProduct(A[0], A[1], B[0], B[1], 20000, net, margin=0.25)
    st = learned.stats
    assert st["capacity"] < st["term_bound"]
    assert st["fallback_rows"] <= 0.05 * st["rows"]
    assert st["class_hits"] >= 0.9 * st["rows"]
    assert scratch_bytes(learned) < scratch_bytes(plain)


@pytest.mark.parametrize("mode", ["untrained_zero_margin", "trained"])
def test_oneshot_product_matches_oracle(sdl, orc, mode):
    """The learned one-shot pass (structure and values of a new pattern in one pass,
    no refill plan) against the oracle: every row class (warp rows, CTA rows, rows
    beyond 8192 terms), rows that overflow their predicted capacity (an untrained
    network with no margin forces many) redone exactly; then the plan is completed
    and a refill with new values equals the plain product's, bit for bit."""
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Product
    from sparsediff_linalg_b200.learned import LearnedFilledProduct, Mlp
    if mode == "trained":
        net, _, _ = _train(sdl, seeds=(30, 31), epochs=6)
        margin = 0.25
    else:
        # a network that predicts no outputs at all: every row gets the minimum
        # capacity (8 slots) and every longer row overflows and is redone exactly
        net, margin = Mlp(seed=9), 0.0
        p = np.zeros(mo.NPARAMS, np.float32)
        p[-4] = -30.0                                   # bias of the row-nnz output
        net.set_params(p)
    A, B = _skewed(77)
    n = 20000
    Q = LearnedFilledProduct(A[0], A[1], B[0], B[1], n, net, A[2], None, B[2], margin=margin)
    assert not Q.plan_ready()
    lens = np.diff(Q.Cp.cpu().numpy())
    ub = np.diff(A[0].cpu().numpy())
    assert lens.max() > 8192 or ub.max() > 0
    hA = tuple(t.cpu().numpy() for t in A) + (n, n)
    hB = tuple(t.cpu().numpy() for t in B) + (n, n)
    want = parallel.spgemm(hA, hB)
    res = parallel.compare_csr((Q.Cp.cpu().numpy(), Q.Ci.cpu().numpy(), Q.values.cpu().numpy()), want)
    assert res["structure_equal"] and res["bit_identical"], res
    if mode != "trained":
        assert Q.stats["fallback_rows"] > 0
    # a refill needs the plan
    cx = torch.empty(Q.nnz, dtype=torch.float64, device="cuda")
    with pytest.raises(Exception):
        Q.fill(A[2], None, B[2], cx)
    Q.complete_plan()
    assert Q.plan_ready()
    P = Product(A[0], A[1], B[0], B[1], n)
    ax = torch.randn(A[2].numel(), dtype=torch.float64, device="cuda")
    bx = torch.randn(B[2].numel(), dtype=torch.float64, device="cuda")
    cp = torch.empty(P.nnz, dtype=torch.float64, device="cuda")
    Q.fill(ax, None, bx, cx)
    P.fill(ax, None, bx, cp)
    torch.cuda.synchronize()
    assert torch.equal(cx.view(torch.int64), cp.view(torch.int64))


def test_oneshot_btda_with_value_map_and_d(sdl, orc):
    """B^T D A through the one-shot pass: L is B's CSC read through the CSR positions
    (L_map) and every entry value is L.x * d[k], as in the refill."""
    import torch
    from oracle import parallel
    from sparsediff_linalg_b200.device import Transpose
    from sparsediff_linalg_b200.learned import LearnedFilledProduct, Mlp
    rng = np.random.default_rng(55)
    m, nA, nB = 30000, 9000, 2000
    A = wl.fixed_rowlen_csr(m, nA, 6, rng)
    # B's columns drawn with skewed popularity, so the rows of C (B's columns) span
    # every class: a few columns hold thousands of entries (over 8192 terms), most few
    pop = 1.0 / np.arange(1, nB + 1) ** 1.1
    pop /= pop.sum()
    ent = np.unique(np.stack([np.repeat(np.arange(m), 4), rng.choice(nB, 4 * m, p=pop)], 1), axis=0)
    Bp = np.zeros(m + 1, np.int32)
    np.add.at(Bp, ent[:, 0] + 1, 1)
    B = (np.cumsum(Bp).astype(np.int32), ent[:, 1].astype(np.int32), rng.standard_normal(len(ent)), m, nB)
    d = rng.uniform(0.1, 10, m)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    Tr = Transpose(T(B[0]), T(B[1]), m, nB)
    net = Mlp(seed=4)
    Q = LearnedFilledProduct(Tr.Tp, Tr.Ti, T(A[0]), T(A[1]), nA, net, T(B[2]), T(d), T(A[2]), margin=0.1,
                             L_map=Tr.src)
    want = parallel.btda(A, B, d)
    res = parallel.compare_csr((Q.Cp.cpu().numpy(), Q.Ci.cpu().numpy(), Q.values.cpu().numpy()), want)
    assert res["structure_equal"] and res["bit_identical"], res
