"""CPU FP64 restatement of the learned row scheduler's network (test
infrastructure): the loss and its gradient, to check the CUDA training kernels.

Layout (matches the library): params = [W1 (32x8), b1 (32), W2 (32x32), b2 (32),
W3 (4x32), b3 (4)], row-major W[out][in]; outputs y = [log1p(nnz) estimate, three
class logits]; per-sample loss 0.5 * (y0 - t0)^2 + cross-entropy(y1..3, class);
the reported loss and gradient are means over the samples."""
import numpy as np

IN, H, OUT = 8, 32, 4
SIZES = [(H, IN), (H,), (H, H), (H,), (OUT, H), (OUT,)]
NPARAMS = sum(int(np.prod(s)) for s in SIZES)


def unpack(p):
    out, at = [], 0
    for s in SIZES:
        k = int(np.prod(s))
        out.append(np.asarray(p[at:at + k], np.float64).reshape(s))
        at += k
    return out


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3.T + b3
    return y, (z1, h1, z2, h2)


def loss_and_grad(p, x, t):
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    n = x.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(p)
    y, (z1, h1, z2, h2) = forward(p, x)
    e = y[:, 0] - t[:, 0]
    lg = y[:, 1:]
    lg = lg - lg.max(axis=1, keepdims=True)
    pr = np.exp(lg)
    pr /= pr.sum(axis=1, keepdims=True)
    c = t[:, 1].astype(int)
    loss = np.mean(0.5 * e * e - np.log(np.maximum(pr[np.arange(n), c], 1e-30)))
    dy = np.zeros_like(y)
    dy[:, 0] = e / n
    oh = np.zeros_like(pr)
    oh[np.arange(n), c] = 1.0
    dy[:, 1:] = (pr - oh) / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dz2 = (dy @ W3) * (z2 > 0)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
