"""The CPU oracle of the learned scheduler's network, pinned by finite differences."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mo.NPARAMS) * 0.3
    x = rng.standard_normal((64, 8))
    t = np.stack([rng.uniform(0, 5, 64), rng.integers(0, 3, 64)], 1)
    loss, g = mo.loss_and_grad(p, x, t)
    eps = 1e-6
    for k in rng.choice(mo.NPARAMS, 40, replace=False):
        q = p.copy()
        q[k] += eps
        l2, _ = mo.loss_and_grad(q, x, t)
        q[k] -= 2 * eps
        l1, _ = mo.loss_and_grad(q, x, t)
        fd = (l2 - l1) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(g[k]), (k, fd, g[k])
