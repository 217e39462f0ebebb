"""ctypes bindings of ``libsparsediff_linalg_b200.so``.

The library exports the upstream C API (``include/sparsediff_linalg/*.h``) plus the
extension API (``include/sparsediff_linalg_cuda.h``). Loading fails loudly when the
library has not been built: there is no Python or CPU fallback for any operation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
# SPARSEDIFF_LINALG_B200_LIB selects another build of the library (e.g. one
# compiled with different tile parameters); default: the in-tree build.
LIB_PATH = Path(os.environ.get("SPARSEDIFF_LINALG_B200_LIB", str(PKG / "libsparsediff_linalg_b200.so")))

c_int_p = C.POINTER(C.c_int)
c_double_p = C.POINTER(C.c_double)


class CSR_matrix(C.Structure):
    """Layout of ``CSR_matrix`` (upstream include/sparsediff_linalg/CSR_matrix.h:31-39)."""
    _fields_ = [("p", c_int_p), ("i", c_int_p), ("x", c_double_p),
                ("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int)]


class CSC_matrix(C.Structure):
    """Layout of ``CSC_matrix`` (upstream include/sparsediff_linalg/CSC_matrix.h:33-41)."""
    _fields_ = [("p", c_int_p), ("i", c_int_p), ("x", c_double_p),
                ("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int)]


class COO_matrix(C.Structure):
    """Layout of ``COO_matrix`` (upstream include/sparsediff_linalg/COO_matrix.h:35-44)."""
    _fields_ = [("rows", c_int_p), ("cols", c_int_p), ("x", c_double_p),
                ("value_map", c_int_p), ("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int)]


class matrix(C.Structure):
    """Layout of the polymorphic ``matrix`` handle (upstream matrix.h:64-88)."""
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int), ("x", c_double_p),
                ("kind", C.c_int), ("values_version", C.c_uint64),
                ("to_csr", C.c_void_p), ("row_gather_alloc", C.c_void_p),
                ("row_gather_fill_values", C.c_void_p), ("row_reduce_alloc", C.c_void_p),
                ("row_reduce_fill_values", C.c_void_p)]


class sdl_product_desc(C.Structure):
    _fields_ = [("Lp", C.c_void_p), ("Li", C.c_void_p), ("L_map", C.c_void_p),
                ("L_m", C.c_int), ("L_nnz", C.c_int), ("blocks", C.c_int),
                ("Ap", C.c_void_p), ("Ai", C.c_void_p),
                ("A_m", C.c_int), ("A_n", C.c_int), ("A_nnz", C.c_int)]


CSR_p = C.POINTER(CSR_matrix)
CSC_p = C.POINTER(CSC_matrix)
COO_p = C.POINTER(COO_matrix)
matrix_p = C.POINTER(matrix)
vp = C.c_void_p

# name -> (restype, argtypes); shared by the product library and, for the upstream
# subset, by the test-side reference build.
UPSTREAM_SIGNATURES = {
    "new_CSR_matrix": (CSR_p, [C.c_int, C.c_int, C.c_int]),
    "new_csr": (CSR_p, [CSR_p]),
    "free_CSR_matrix": (None, [CSR_p]),
    "copy_CSR_matrix": (None, [CSR_p, CSR_p]),
    "CSR_trim": (None, [CSR_p]),
    "transpose": (CSR_p, [CSR_p, c_int_p]),
    "AT_alloc": (CSR_p, [CSR_p, c_int_p]),
    "AT_fill_values": (None, [CSR_p, CSR_p, c_int_p]),
    "new_CSC_matrix": (CSC_p, [C.c_int, C.c_int, C.c_int]),
    "free_CSC_matrix": (None, [CSC_p]),
    "BTA_alloc": (CSR_p, [CSR_p, CSC_p]),
    "BTDA_fill_values": (None, [CSR_p, CSC_p, vp, vp, CSR_p]),
    "csr_to_csc_alloc": (CSC_p, [CSR_p, c_int_p]),
    "csr_to_csc_fill_values": (None, [CSR_p, CSC_p, c_int_p]),
    "csc_to_csr_alloc": (CSR_p, [CSC_p, c_int_p]),
    "csc_to_csr_fill_values": (None, [CSC_p, CSR_p, c_int_p]),
    "new_COO_matrix": (COO_p, [CSR_p]),
    "new_COO_matrix_lower_triangular": (COO_p, [CSR_p]),
    "refresh_lower_triangular_coo": (None, [COO_p, vp]),
    "free_COO_matrix": (None, [COO_p]),
}

EXTENSION_SIGNATURES = {
    "sdl_last_status": (C.c_int, []),
    "sdl_last_error": (C.c_char_p, []),
    "sdl_clear_error": (None, []),
    "sdl_set_fatal_errors": (None, [C.c_int]),
    "sdl_device_available": (C.c_int, []),
    "sdl_device_alloc_count": (C.c_ulonglong, []),
    "sdl_release_cached_memory": (None, []),
    "sdl_kernel_launch_count": (C.c_ulonglong, []),
    "sdl_stream": (vp, []),
    "sdl_synchronize": (C.c_int, []),
    "sdl_free": (None, [vp]),
    "sdl_product_create": (C.c_int, [C.POINTER(sdl_product_desc), vp, C.POINTER(vp)]),
    "sdl_product_info": (C.c_int, [vp, c_int_p, c_int_p, c_int_p, C.POINTER(C.c_longlong),
                                   C.POINTER(vp), C.POINTER(vp)]),
    "sdl_product_fill": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "sdl_product_autotune": (C.c_int, [vp, C.c_int, vp]),
    "sdl_product_tuning": (C.c_int, [vp, c_int_p, c_int_p, c_int_p, c_int_p, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), c_int_p, C.POINTER(C.c_double)]),
    "sdl_product_refill_shape": (C.c_int, [vp, c_int_p, c_int_p]),
    "sdl_product_create_learned_filled": (C.c_int, [C.POINTER(sdl_product_desc), vp, C.c_float, vp, vp, vp, vp,
                                                    C.POINTER(vp), vp]),
    "sdl_product_values": (C.c_int, [vp, vp]),
    "sdl_product_complete_plan": (C.c_int, [vp, vp]),
    "sdl_product_plan_ready": (C.c_int, [vp, c_int_p]),
    "sdl_product_set_refill_pipe": (C.c_int, [vp, C.c_int, c_int_p]),
    "sdl_product_refill_pipe_used": (C.c_int, [vp, c_int_p]),
    "sdl_product_set_refill_staged": (C.c_int, [vp, C.c_int, c_int_p]),
    "sdl_product_refill_staged_used": (C.c_int, [vp, c_int_p]),
    "sdl_batch_autotune": (C.c_int, [vp, C.c_int, vp, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
    "sdl_product_apply_tuned": (C.c_int, [vp, c_int_p, vp]),
    "sdl_product_pattern_key": (C.c_int, [vp, C.c_char_p, C.c_int, vp]),
    "sdl_tune_table_save": (C.c_int, [C.c_char_p]),
    "sdl_tune_table_load": (C.c_int, [C.c_char_p, c_int_p]),
    "sdl_tune_table_clear": (C.c_int, []),
    "sdl_tune_table_size": (C.c_int, [c_int_p]),
    "sdl_product_replan": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]),
    "sdl_product_destroy": (None, [vp]),
    "sdl_product_fill_noalloc": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "sdl_batch_create": (C.c_int, [C.POINTER(vp), C.c_int, vp, C.POINTER(vp)]),
    "sdl_batch_bind": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "sdl_batch_refill": (C.c_int, [vp, vp]),
    "sdl_batch_set_group_bytes": (C.c_int, [vp, C.c_longlong]),
    "sdl_batch_groups": (C.c_int, [vp, c_int_p]),
    "sdl_batch_refill_unbatched": (C.c_int, [vp, vp]),
    "sdl_batch_info": (C.c_int, [vp, c_int_p, c_int_p, C.POINTER(C.c_longlong)]),
    "sdl_batch_destroy": (None, [vp]),
    "sdl_mlp_create": (C.c_int, [C.c_ulonglong, C.POINTER(vp)]),
    "sdl_mlp_destroy": (None, [vp]),
    "sdl_mlp_get_params": (C.c_int, [vp, vp]),
    "sdl_mlp_set_params": (C.c_int, [vp, vp]),
    "sdl_product_row_stats": (C.c_int, [vp, vp, vp, vp]),
    "sdl_mlp_gradient": (C.c_int, [vp, vp, vp, C.c_int, vp, C.POINTER(C.c_float)]),
    "sdl_mlp_train": (C.c_int, [vp, vp, vp, C.c_longlong, C.c_int, C.c_int, C.c_float, C.c_ulonglong,
                                C.POINTER(C.c_float)]),
    "sdl_mlp_predict": (C.c_int, [vp, vp, C.c_longlong, vp, vp]),
    "sdl_product_create_learned": (C.c_int, [C.POINTER(sdl_product_desc), vp, C.c_float, vp, C.POINTER(vp),
                                             vp]),
    "sdl_product_scratch_bytes": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
    "sdl_transpose_create": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, vp, C.POINTER(vp)]),
    "sdl_transpose_info": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "sdl_transpose_fill": (C.c_int, [vp, vp, vp, vp]),
    "sdl_transpose_destroy": (None, [vp]),
    "sdl_coalesce_create": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, vp, C.POINTER(vp)]),
    "sdl_coalesce_info": (C.c_int, [vp, c_int_p, C.POINTER(vp), C.POINTER(vp)]),
    "sdl_coalesce_fill": (C.c_int, [vp, vp, vp, vp]),
    "sdl_coalesce_destroy": (None, [vp]),
    "sdl_blocks_csr_create": (C.c_int, [C.c_int, vp, vp, C.POINTER(vp), vp, vp, C.c_int, C.c_int, C.c_int,
                                        vp, C.POINTER(vp)]),
    "sdl_blocks_csr_info": (C.c_int, [vp, c_int_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sdl_blocks_csr_block": (C.c_int, [vp, C.c_int, c_int_p, c_int_p, c_int_p, C.POINTER(vp)]),
    "sdl_blocks_csr_fill": (C.c_int, [vp, vp, vp, vp, vp]),
    "sdl_blocks_csr_destroy": (None, [vp]),
    "sdl_blocks_ata_create": (C.c_int, [C.c_int, vp, vp, C.POINTER(vp), C.POINTER(vp), C.c_int, C.c_int, vp,
                                        C.POINTER(vp)]),
    "sdl_blocks_ata_info": (C.c_int, [vp, c_int_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sdl_blocks_ata_block": (C.c_int, [vp, C.c_int, c_int_p, c_int_p, C.POINTER(vp), C.POINTER(vp)]),
    "sdl_blocks_ata_fill": (C.c_int, [vp, vp, vp, vp, vp]),
    "sdl_blocks_ata_destroy": (None, [vp]),
    "COO_coalesce_alloc": (CSR_p, [COO_p]),
    "COO_coalesce_fill_values": (None, [COO_p, CSR_p]),
}


def bind(lib: C.CDLL, sigs: dict) -> C.CDLL:
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded CUDA library. Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built: run `python -m sparsediff_linalg_b200._build` "
                "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        bind(L, UPSTREAM_SIGNATURES)
        bind(L, EXTENSION_SIGNATURES)
        _LIB = L
    return _LIB


class SDLError(RuntimeError):
    pass


def check(status: int) -> None:
    if status != 0:
        msg = lib().sdl_last_error()
        raise SDLError(f"status {status}: {msg.decode() if msg else ''}")
