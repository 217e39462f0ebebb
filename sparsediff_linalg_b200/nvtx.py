"""NVTX ranges for host-side phases (named spans on an Nsight Systems timeline).

The library marks its own phases (symbolic pass, refill, host transfers) with
NVTX ranges in C++; this helper marks the caller's phases around them. Without a
CUDA build of torch it is a no-op.
"""
from __future__ import annotations

import contextlib


@contextlib.contextmanager
def range(name: str):  # noqa: A001 - mirrors nvtx's own name
    try:
        import torch
        push, pop = torch.cuda.nvtx.range_push, torch.cuda.nvtx.range_pop
        push(name)
    except Exception:
        push = pop = None
    try:
        yield
    finally:
        if pop is not None:
            try:
                pop()
            except Exception:
                pass
