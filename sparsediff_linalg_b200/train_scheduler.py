"""Train the learned row scheduler on the row statistics the exact symbolic pass
produces for seeded Zipf-skewed products (C = A B, A and B with Zipf(1.5) row
lengths), and save its parameters (1476 float32, little-endian).

    python -m sparsediff_linalg_b200.train_scheduler --out weights.bin [--matrices 200]

Matrices are m x m with ~20 nnz per row on average (the full-size configuration's
density) and row lengths capped at m / 20; the features are scale-aware (they
include log n), so a network trained on smaller matrices transfers to 1M x 1M.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def collect(matrices=200, m=40_000, rows_per_matrix=8_000, seed0=1000):
    import torch
    from . import workloads as wl
    from .device import Product
    from .learned import row_stats
    feats, labels = [], []
    g = torch.Generator(device="cuda")
    g.manual_seed(seed0)
    for k in range(matrices):
        (Ap, Ai, _), (Bp, Bi, _), _ = wl.skewed_device(seed=seed0 + k, m=m, n=m, target=20 * m,
                                                       cap=max(50, m // 20))
        P = Product(Ap, Ai, Bp, Bi, m)
        f, l = row_stats(P)
        sel = torch.randperm(m, generator=g, device="cuda")[:rows_per_matrix]
        feats.append(f[sel])
        labels.append(l[sel])
        del P
    return torch.cat(feats).contiguous(), torch.cat(labels).contiguous()


def train(matrices=200, epochs=8, seed=0, **kw):
    from .learned import Mlp
    t0 = time.perf_counter()
    F, L = collect(matrices=matrices, **kw)
    t_collect = time.perf_counter() - t0
    net = Mlp(seed=seed)
    first, _ = net.gradient(F, L)
    t0 = time.perf_counter()
    last = net.train(F, L, epochs=epochs, batch=8192, lr=3e-3, seed=seed)
    t_train = time.perf_counter() - t0
    return net, {"samples": int(F.shape[0]), "matrices": matrices, "loss_initial": round(first, 4),
                 "loss_final": round(last, 4), "collect_s": round(t_collect, 2),
                 "train_s": round(t_train, 2), "epochs": epochs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--matrices", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=8)
    a = ap.parse_args()
    net, info = train(matrices=a.matrices, epochs=a.epochs)
    net.params().astype("<f4").tofile(a.out)
    print(info)


if __name__ == "__main__":
    main()
