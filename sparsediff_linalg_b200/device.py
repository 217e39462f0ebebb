"""Device-resident wrappers (torch tensors in HBM) over the extension C API.

Torch provides device memory and streams only; every computation is a kernel of
``libsparsediff_linalg_b200.so``.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import check, lib, sdl_product_desc


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    """cudaStream_t of a torch stream. torch's legacy default stream has handle 0,
    which the C API reads as "the library's stream", so it is passed as
    cudaStreamLegacy (0x1) instead: work is then ordered with torch's kernels and
    events recorded on that stream bracket it."""
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream or 1)


class _DevView:
    """__cuda_array_interface__ over a library-owned device array."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {
            "shape": (int(n),), "typestr": typestr, "data": (int(ptr or 0), False), "version": 3,
            "strides": None,
        }


def _as_tensor(ptr, n, typestr="<i4"):
    if n == 0:
        return torch.zeros(0, dtype=torch.int32, device="cuda")
    return torch.as_tensor(_DevView(ptr, n, typestr), device="cuda")


class Product:
    """C = kron(I_blocks, L) diag(d) A with device-resident operands.

    L is given by rows (Lp, Li) over the rows of A (within a block); L_map (optional)
    makes L's value of entry ii equal Lx[L_map[ii]]. The structure tensors must stay
    alive (they are referenced, not copied)."""

    def __init__(self, Lp, Li, Ap, Ai, A_n, L_map=None, blocks=1, stream=None):
        L = lib()
        self._keep = (Lp, Li, Ap, Ai, L_map)
        desc = sdl_product_desc(
            _ptr(Lp).value, _ptr(Li).value, _ptr(L_map).value if L_map is not None else None,
            Lp.numel() - 1, Li.numel(), blocks, _ptr(Ap).value, _ptr(Ai).value,
            Ap.numel() - 1, A_n, Ai.numel())
        h = C.c_void_p()
        check(L.sdl_product_create(C.byref(desc), _stream(stream), C.byref(h)))
        self._init_from_handle(h)

    def _init_from_handle(self, h):
        L = lib()
        self.handle = h
        m, n, nnz = C.c_int(), C.c_int(), C.c_int()
        terms = C.c_longlong()
        cp, ci = C.c_void_p(), C.c_void_p()
        check(L.sdl_product_info(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(terms),
                                 C.byref(cp), C.byref(ci)))
        self.m, self.n, self.nnz, self.terms = m.value, n.value, nnz.value, terms.value
        self.Cp = _as_tensor(cp.value, self.m + 1)
        self.Ci = _as_tensor(ci.value, self.nnz)

    def fill(self, Lx, d, Ax, Cx, stream=None):
        check(lib().sdl_product_fill(self.handle, _ptr(Lx), _ptr(d), _ptr(Ax), _ptr(Cx),
                                     _stream(stream)))

    def autotune(self, reps=5, stream=None):
        """Re-plan for this pattern (sdl_product_autotune); returns tuning()."""
        check(lib().sdl_product_autotune(self.handle, reps, _stream(stream)))
        self._init_from_handle(self.handle)
        return self.tuning()

    def replan(self, tile_budget=0, tile_max_terms=0, refill_threads=256, refill_ctas_per_sm=0, stream=None):
        """Re-plan with a given refill configuration (sdl_product_replan)."""
        check(lib().sdl_product_replan(self.handle, tile_budget, tile_max_terms, refill_threads,
                                       refill_ctas_per_sm, _stream(stream)))
        self._init_from_handle(self.handle)

    def apply_tuned(self, stream=None):
        """Re-plan with the tuning table's configuration for this pattern (True if
        the table had one)."""
        found = C.c_int()
        check(lib().sdl_product_apply_tuned(self.handle, C.byref(found), _stream(stream)))
        if found.value:
            self._init_from_handle(self.handle)
        return bool(found.value)

    def pattern_key(self, stream=None):
        buf = C.create_string_buffer(512)
        check(lib().sdl_product_pattern_key(self.handle, buf, 512, _stream(stream)))
        return buf.value.decode()

    def refill_pipelined(self):
        used = C.c_int()
        check(lib().sdl_product_refill_pipe_used(self.handle, C.byref(used)))
        return bool(used.value)

    def set_refill_pipe(self, on):
        """Pipelined (True) or direct (False) tile refill; returns whether the
        pipelined refill will run for this plan."""
        used = C.c_int()
        check(lib().sdl_product_set_refill_pipe(self.handle, 1 if on else 0, C.byref(used)))
        return bool(used.value)

    def refill_staged(self):
        used = C.c_int()
        check(lib().sdl_product_refill_staged_used(self.handle, C.byref(used)))
        return bool(used.value)

    def set_refill_staged(self, on):
        """Staged (True: tile words and entry records bulk-copied into shared
        memory a tile ahead) or plain (False) direct tile refill; returns whether the
        staged refill will run for this plan."""
        used = C.c_int()
        check(lib().sdl_product_set_refill_staged(self.handle, 1 if on else 0, C.byref(used)))
        return bool(used.value)

    def refill_shape(self):
        th, tm = C.c_int(), C.c_int()
        check(lib().sdl_product_refill_shape(self.handle, C.byref(th), C.byref(tm)))
        return th.value, tm.value

    def tuning(self):
        """The plan's configuration and what the autotuner measured."""
        i = [C.c_int() for _ in range(5)]
        f = [C.c_double() for _ in range(3)]
        check(lib().sdl_product_tuning(self.handle, C.byref(i[0]), C.byref(i[1]), C.byref(i[2]),
                                       C.byref(i[3]), C.byref(f[0]), C.byref(f[1]), C.byref(i[4]),
                                       C.byref(f[2])))
        th, tm = C.c_int(), C.c_int()
        check(lib().sdl_product_refill_shape(self.handle, C.byref(th), C.byref(tm)))
        kind = "pipelined" if self.refill_pipelined() else "staged" if self.refill_staged() else "direct"
        return {"refill": kind, "warp_max_terms": i[0].value, "rows_per_cta_warp": i[1].value, "tile_budget": i[2].value,
                "refill_ctas_per_sm": i[3].value, "refill_threads": th.value, "tile_max_terms": tm.value,
                "refill_us": round(f[0].value, 2),
                "default_refill_us": round(f[1].value, 2), "candidates": i[4].value,
                "tune_ms": round(f[2].value, 1)}

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_product_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class Transpose:
    """Stable transpose plan of a device compressed structure (rows x cols)."""

    def __init__(self, p, idx, rows, cols, stream=None):
        L = lib()
        self._keep = (p, idx)
        h = C.c_void_p()
        nnz = idx.numel()
        check(L.sdl_transpose_create(_ptr(p), _ptr(idx), rows, cols, nnz, _stream(stream), C.byref(h)))
        self.handle = h
        tp, ti, src = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(L.sdl_transpose_info(h, C.byref(tp), C.byref(ti), C.byref(src)))
        self.nnz = nnz
        self.Tp = _as_tensor(tp.value, cols + 1)
        self.Ti = _as_tensor(ti.value, nnz)
        self.src = _as_tensor(src.value, nnz)

    def fill(self, x, Tx, stream=None):
        check(lib().sdl_transpose_fill(self.handle, _ptr(x), _ptr(Tx), _stream(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_transpose_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class Coalesce:
    """Duplicate-coalescing plan of device COO triplets (rows, cols) into an m x n CSR."""

    def __init__(self, rows, cols, m, n, stream=None):
        L = lib()
        h = C.c_void_p()
        check(L.sdl_coalesce_create(_ptr(rows), _ptr(cols), rows.numel(), m, n, _stream(stream),
                                    C.byref(h)))
        self.handle = h
        nnz = C.c_int()
        cp, ci = C.c_void_p(), C.c_void_p()
        check(L.sdl_coalesce_info(h, C.byref(nnz), C.byref(cp), C.byref(ci)))
        self.m, self.n, self.nnz = m, n, nnz.value
        self.Cp = _as_tensor(cp.value, m + 1)
        self.Ci = _as_tensor(ci.value, self.nnz)

    def fill(self, x, Cx, stream=None):
        check(lib().sdl_coalesce_fill(self.handle, _ptr(x), _ptr(Cx), _stream(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_coalesce_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class BlocksCsr:
    """C_k = B_k S[col_perm_k, :] for dense blocks B_k (m0[k] x n0[k], a stacked_pd's
    blocks) and a sparse CSR S (sdl_blocks_csr_*). The structure is taken from host
    arrays; fill() works on device tensors: B_vals (source blocks in order, each
    row-major), S_x, and C_vals (output blocks in order, each m0 x n0_C row-major)."""

    def __init__(self, m0, n0, col_perms, Sp, Si, S_m, S_n, keep_empty=False, stream=None):
        import numpy as np
        L = lib()
        nb = len(m0)
        self._m0 = np.ascontiguousarray(m0, np.int32)
        self._n0 = np.ascontiguousarray(n0, np.int32)
        self._perms = [np.ascontiguousarray(c, np.int32) for c in col_perms]
        arr = (C.c_void_p * max(1, nb))(*[c.ctypes.data for c in self._perms])
        self._Sp = np.ascontiguousarray(Sp, np.int32)
        self._Si = np.ascontiguousarray(Si, np.int32)
        h = C.c_void_p()
        check(L.sdl_blocks_csr_create(nb, self._m0.ctypes.data, self._n0.ctypes.data, arr,
                                      self._Sp.ctypes.data, self._Si.ctypes.data, S_m, S_n,
                                      1 if keep_empty else 0, _stream(stream), C.byref(h)))
        self.handle = h
        ob, cv, bv = C.c_int(), C.c_longlong(), C.c_longlong()
        check(L.sdl_blocks_csr_info(h, C.byref(ob), C.byref(cv), C.byref(bv)))
        self.out_blocks, self.c_values, self.b_values = ob.value, cv.value, bv.value
        self.blocks = []
        for k in range(self.out_blocks):
            src, m, n0c, cp = C.c_int(), C.c_int(), C.c_int(), C.c_void_p()
            check(L.sdl_blocks_csr_block(h, k, C.byref(src), C.byref(m), C.byref(n0c), C.byref(cp)))
            if n0c.value > 0:
                perm = np.ctypeslib.as_array(C.cast(cp, C.POINTER(C.c_int)), shape=(n0c.value,)).copy()
            else:
                perm = np.zeros(0, np.int32)
            self.blocks.append((src.value, m.value, n0c.value, perm))

    def fill(self, B_vals, S_x, C_vals, stream=None):
        check(lib().sdl_blocks_csr_fill(self.handle, _ptr(B_vals), _ptr(S_x), _ptr(C_vals),
                                        _stream(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_blocks_csr_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class BlocksAta:
    """A^T diag(d) A of dense blocks (m0[k] x n0[k] at rows row_perms[k] of m and
    columns col_perms[k] of n) on the FP64 tensor cores, coalesced as upstream's
    stacked_pd (sdl_blocks_ata_*). fill() works on device tensors: X_vals (blocks in
    order, row-major), d (m values or None), C_vals (output blocks in order)."""

    def __init__(self, m0, n0, row_perms, col_perms, m, n, stream=None):
        import numpy as np
        L = lib()
        nb = len(m0)
        self._m0 = np.ascontiguousarray(m0, np.int32)
        self._n0 = np.ascontiguousarray(n0, np.int32)
        self._rp = [np.ascontiguousarray(r, np.int32) for r in row_perms]
        self._cp = [np.ascontiguousarray(c, np.int32) for c in col_perms]
        ra = (C.c_void_p * max(1, nb))(*[r.ctypes.data for r in self._rp])
        ca = (C.c_void_p * max(1, nb))(*[c.ctypes.data for c in self._cp])
        h = C.c_void_p()
        check(L.sdl_blocks_ata_create(nb, self._m0.ctypes.data, self._n0.ctypes.data, ra, ca, m, n,
                                      _stream(stream), C.byref(h)))
        self.handle = h
        ob, cv, xv = C.c_int(), C.c_longlong(), C.c_longlong()
        check(L.sdl_blocks_ata_info(h, C.byref(ob), C.byref(cv), C.byref(xv)))
        self.out_blocks, self.c_values, self.x_values = ob.value, cv.value, xv.value
        self.blocks = []
        for k in range(self.out_blocks):
            mm, nn, rr, cc = C.c_int(), C.c_int(), C.c_void_p(), C.c_void_p()
            check(L.sdl_blocks_ata_block(h, k, C.byref(mm), C.byref(nn), C.byref(rr), C.byref(cc)))
            rows = np.ctypeslib.as_array(C.cast(rr, C.POINTER(C.c_int)), shape=(mm.value,)).copy() \
                if mm.value else np.zeros(0, np.int32)
            cols = np.ctypeslib.as_array(C.cast(cc, C.POINTER(C.c_int)), shape=(nn.value,)).copy() \
                if nn.value else np.zeros(0, np.int32)
            self.blocks.append((rows, cols))

    def fill(self, X_vals, d, C_vals, stream=None):
        check(lib().sdl_blocks_ata_fill(self.handle, _ptr(X_vals), _ptr(d), _ptr(C_vals), _stream(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_blocks_ata_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class Batch:
    """Batched refill of many products: a few grouped persistent launches over all
    their tiles, replayed from a CUDA graph (sdl_batch_*)."""

    def __init__(self, products, stream=None):
        L = lib()
        self._keep = list(products)
        arr = (C.c_void_p * max(1, len(products)))(*[p.handle for p in products])
        h = C.c_void_p()
        check(L.sdl_batch_create(arr, len(products), _stream(stream), C.byref(h)))
        self.handle = h
        t, b, n = C.c_int(), C.c_int(), C.c_longlong()
        check(L.sdl_batch_info(h, C.byref(t), C.byref(b), C.byref(n)))
        self.tiles, self.big_rows, self.terms = t.value, b.value, n.value
        self._bound = {}

    def set_group_bytes(self, nbytes):
        """Bytes of entry values and records per product group (0: one group);
        only before the first refill."""
        check(lib().sdl_batch_set_group_bytes(self.handle, int(nbytes)))

    @property
    def groups(self):
        g = C.c_int()
        check(lib().sdl_batch_groups(self.handle, C.byref(g)))
        return g.value

    def bind(self, i, Lx, d, Ax, Cx):
        self._bound[i] = (Lx, d, Ax, Cx)
        check(lib().sdl_batch_bind(self.handle, i, _ptr(Lx), _ptr(d), _ptr(Ax), _ptr(Cx)))

    def autotune(self, reps=3, stream=None):
        """Times the candidate group sizes before the first refill and keeps the
        fastest (sdl_batch_autotune). Returns (group bytes, ms per refill)."""
        gb, ms = C.c_longlong(), C.c_double()
        check(lib().sdl_batch_autotune(self.handle, reps, _stream(stream), C.byref(gb), C.byref(ms)))
        return gb.value, ms.value

    def refill(self, stream=None):
        check(lib().sdl_batch_refill(self.handle, _stream(stream)))

    def refill_unbatched(self, stream=None):
        check(lib().sdl_batch_refill_unbatched(self.handle, _stream(stream)))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().sdl_batch_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def btda_product(A_p, A_i, A_n, B_p, B_i, B_n, stream=None):
    """Device plan of C = B^T D A with A, B given as device CSR structures: B's CSC is
    built by a transpose plan and its values are read through the CSR positions
    (no CSC value refresh). Returns (product, transpose)."""
    m = A_p.numel() - 1
    T = Transpose(B_p, B_i, m, B_n, stream=stream)
    P = Product(T.Tp, T.Ti, A_p, A_i, A_n, L_map=T.src, stream=stream)
    P._owner = T  # the product's L arrays belong to the transpose plan: keep it alive with P
    return P, T


def btda_product_rows(A_p, A_i, A_n, B_p, B_i, B_n, r0, r1, transpose=None, stream=None):
    """Rows r0 .. r1 - 1 of C = B^T D A (columns r0 .. r1 - 1 of B) as a product of
    their own: L is the slice of B's CSC over those columns, A is whole. Its fill
    takes the full value arrays (B.x, d, A.x) and writes exactly those rows of C, in
    the bits of the whole product. `transpose` shares B's transpose plan between the
    slices (built here when None). Returns (product, transpose)."""
    m = A_p.numel() - 1
    T = transpose if transpose is not None else Transpose(B_p, B_i, m, B_n, stream=stream)
    if not (0 <= r0 <= r1 <= B_n):
        raise ValueError("row range outside the product")
    tp = T.Tp[r0:r1 + 1].cpu()
    s0, s1 = int(tp[0]), int(tp[-1])
    Lp = torch.as_tensor((tp - s0).to(torch.int32), device=A_p.device)
    P = Product(Lp, T.Ti[s0:s1], A_p, A_i, A_n, L_map=T.src[s0:s1], stream=stream)
    P._owner = T
    return P, T


def spgemm_product_rows(A_p, A_i, B_p, B_i, B_n, r0, r1, stream=None):
    """Rows r0 .. r1 - 1 of C = A B as a product of their own: L is the slice of A's
    rows, B is whole. Returns (product, (s0, s1)): its fill takes A.x[s0:s1] as the
    L values and the whole B.x, and writes exactly those rows of C, in the bits of
    the whole product."""
    m = A_p.numel() - 1
    if not (0 <= r0 <= r1 <= m):
        raise ValueError("row range outside the product")
    ap = A_p[r0:r1 + 1].cpu()
    s0, s1 = int(ap[0]), int(ap[-1])
    Lp = torch.as_tensor((ap - s0).to(torch.int32), device=A_p.device)
    Li = A_i[s0:s1]
    P = Product(Lp, Li, B_p, B_i, B_n, stream=stream)
    return P, (s0, s1)


class KeyGrouping:
    """Stable grouping of positions 0 .. N-1 by int32 keys in [0, nkeys): the
    library's stable transpose of the one-entry-per-row structure. `offsets`
    (nkeys + 1), `perm` (positions in key order, ties in position order),
    `gather(x)` = x[perm] for float64 x (the library's value gather)."""

    def __init__(self, keys, nkeys, stream=None):
        n = int(keys.numel())
        self._p = torch.arange(n + 1, dtype=torch.int32, device=keys.device)
        self._t = Transpose(self._p, keys.contiguous(), n, nkeys, stream=stream)
        self.offsets = self._t.Tp
        self.perm = self._t.src

    def gather(self, x, stream=None):
        out = torch.empty(max(1, int(self.perm.numel())), dtype=torch.float64, device=x.device)
        if self.perm.numel():
            self._t.fill(x.contiguous(), out, stream=stream)
        return out[:int(self.perm.numel())]


def group_by_key(keys, nkeys):
    return KeyGrouping(keys, nkeys)


def tune_table_save(path):
    check(lib().sdl_tune_table_save(str(path).encode()))


def tune_table_load(path):
    n = C.c_int()
    check(lib().sdl_tune_table_load(str(path).encode(), C.byref(n)))
    return n.value


def tune_table_clear():
    check(lib().sdl_tune_table_clear())


def tune_table_size():
    n = C.c_int()
    check(lib().sdl_tune_table_size(C.byref(n)))
    return n.value
