"""The learned row scheduler (sdl_mlp_*, sdl_product_create_learned) from Python."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, sdl_product_desc
from .device import Product, _ptr, _stream

NPARAMS = 1476


class LearnedStats(C.Structure):
    _fields_ = [("rows", C.c_longlong), ("term_bound", C.c_longlong), ("capacity", C.c_longlong),
                ("fallback_rows", C.c_longlong), ("fallback_terms", C.c_longlong),
                ("class_hits", C.c_longlong), ("scratch_bytes", C.c_longlong)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class Mlp:
    def __init__(self, seed=0):
        h = C.c_void_p()
        check(lib().sdl_mlp_create(seed, C.byref(h)))
        self.handle = h

    def params(self):
        out = np.zeros(NPARAMS, np.float32)
        check(lib().sdl_mlp_get_params(self.handle, out.ctypes.data))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == NPARAMS
        check(lib().sdl_mlp_set_params(self.handle, p.ctypes.data))

    def gradient(self, feat, label):
        g = np.zeros(NPARAMS, np.float32)
        loss = C.c_float()
        check(lib().sdl_mlp_gradient(self.handle, _ptr(feat), _ptr(label), feat.shape[0], g.ctypes.data,
                                     C.byref(loss)))
        return loss.value, g

    def train(self, feat, label, epochs=10, batch=4096, lr=3e-3, seed=0):
        loss = C.c_float()
        check(lib().sdl_mlp_train(self.handle, _ptr(feat), _ptr(label), feat.shape[0], epochs, batch, lr,
                                  seed, C.byref(loss)))
        return loss.value

    def predict(self, feat, stream=None):
        import torch
        out = torch.empty((feat.shape[0], 4), dtype=torch.float32, device=feat.device)
        check(lib().sdl_mlp_predict(self.handle, _ptr(feat), feat.shape[0], _ptr(out), _stream(stream)))
        return out

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_mlp_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def row_stats(product, stream=None):
    """(features [rows, 8], labels [rows, 2]) float32 device tensors of a product."""
    import torch
    feat = torch.empty((product.m, 8), dtype=torch.float32, device="cuda")
    label = torch.empty((product.m, 2), dtype=torch.float32, device="cuda")
    check(lib().sdl_product_row_stats(product.handle, _ptr(feat), _ptr(label), _stream(stream)))
    return feat, label


class LearnedProduct(Product):
    """A product built by the learned symbolic pass (same structure as Product)."""

    def __init__(self, Lp, Li, Ap, Ai, A_n, net, margin=0.25, L_map=None, blocks=1, stream=None):
        L = lib()
        self._keep = (Lp, Li, Ap, Ai, L_map, net)
        desc = sdl_product_desc(
            _ptr(Lp).value, _ptr(Li).value, _ptr(L_map).value if L_map is not None else None,
            Lp.numel() - 1, Li.numel(), blocks, _ptr(Ap).value, _ptr(Ai).value,
            Ap.numel() - 1, A_n, Ai.numel())
        h = C.c_void_p()
        st = LearnedStats()
        check(L.sdl_product_create_learned(C.byref(desc), net.handle, margin, _stream(stream), C.byref(h),
                                           C.byref(st)))
        self.stats = st.as_dict()
        self._init_from_handle(h)


class LearnedFilledProduct(Product):
    """A pattern met for the first time: C's structure and values from the learned
    one-shot pass (sdl_product_create_learned_filled). `values` is C.x (device,
    owned by the product); refills need complete_plan() first."""

    def __init__(self, Lp, Li, Ap, Ai, A_n, net, Lx, d, Ax, margin=0.25, L_map=None, blocks=1, stream=None):
        L = lib()
        self._keep = (Lp, Li, Ap, Ai, L_map, net, Lx, d, Ax)
        desc = sdl_product_desc(
            _ptr(Lp).value, _ptr(Li).value, _ptr(L_map).value if L_map is not None else None,
            Lp.numel() - 1, Li.numel(), blocks, _ptr(Ap).value, _ptr(Ai).value,
            Ap.numel() - 1, A_n, Ai.numel())
        h = C.c_void_p()
        st = LearnedStats()
        check(L.sdl_product_create_learned_filled(C.byref(desc), net.handle, margin, _ptr(Lx), _ptr(d), _ptr(Ax),
                                                  _stream(stream), C.byref(h), C.byref(st)))
        self.stats = st.as_dict()
        self._init_from_handle(h)
        cx = C.c_void_p()
        check(L.sdl_product_values(self.handle, C.byref(cx)))
        from .device import _as_tensor
        self.values = _as_tensor(cx.value, self.nnz, "<f8") if self.nnz else None

    def plan_ready(self):
        r = C.c_int()
        check(lib().sdl_product_plan_ready(self.handle, C.byref(r)))
        return bool(r.value)

    def complete_plan(self, stream=None):
        check(lib().sdl_product_complete_plan(self.handle, _stream(stream)))
        self._init_from_handle(self.handle)


def scratch_bytes(product):
    b = C.c_longlong()
    check(lib().sdl_product_scratch_bytes(product.handle, C.byref(b)))
    return b.value
