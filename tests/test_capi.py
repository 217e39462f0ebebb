"""C-ABI boundary checks that need no GPU: the library loads, exports every
function the public headers declare, keeps upstream's struct layouts, and the
host-only constructors behave like upstream's. Without a device, compute entry
points must fail loudly (status / exit), never fall back to the CPU."""
import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import GPU, ROOT
from sparsediff_linalg_b200 import _lib
from sparsediff_linalg_b200.host import HostCSR, csr_from_ptr

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?[\s\*]([A-Za-z_]\w*)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").rglob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = "\n".join(l for l in text.splitlines() if not l.strip().startswith("#"))
        text = text.replace('extern "C" {', "")
        # drop bodies of inline functions and struct definitions
        while True:
            t2 = re.sub(r"\{[^{}]*\}", ";", text)
            if t2 == text:
                break
            text = t2
        for stmt in text.split(";"):
            s = " ".join(stmt.split())
            if not s or s.startswith("typedef") or s.startswith("static") or s.startswith("struct"):
                continue
            m = DECL.search(s)
            if m:
                names.add(m.group(1))
    return names


def test_headers_declare_the_hot_path():
    names = declared_functions()
    for must in ["BTA_alloc", "BTDA_fill_values", "csr_to_csc_alloc", "csc_to_csr_fill_values",
                 "AT_alloc", "transpose", "BTA_matrices_alloc", "BTDA_matrices_fill_values",
                 "BA_matrices_alloc", "ATA_matrices_alloc", "sdl_product_create", "sdl_coalesce_create"]:
        assert must in names, must


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_struct_layouts_match_upstream():
    assert C.sizeof(_lib.CSR_matrix) == 40 and C.sizeof(_lib.CSC_matrix) == 40
    assert C.sizeof(_lib.COO_matrix) == 48
    assert _lib.matrix.values_version.offset == 32 and _lib.matrix.to_csr.offset == 40
    assert C.sizeof(_lib.matrix) == 80


def test_host_constructors():
    L = _lib.lib()
    A = L.new_CSR_matrix(3, 4, 5)
    s = A.contents
    assert (s.m, s.n, s.nnz) == (3, 4, 5)
    assert np.ctypeslib.as_array(s.p, shape=(4,)).tolist() == [0, 0, 0, 0]
    np.ctypeslib.as_array(s.p, shape=(4,))[:] = [0, 2, 2, 3]
    np.ctypeslib.as_array(s.i, shape=(5,))[:] = [0, 3, 1, 0, 0]
    np.ctypeslib.as_array(s.x, shape=(5,))[:] = [1, 2, 3, 0, 0]
    B = L.new_csr(A)
    L.CSR_trim(B)
    assert B.contents.nnz == 3
    p, i, x, m, n = csr_from_ptr(B)
    assert p.tolist() == [0, 2, 2, 3] and i.tolist() == [0, 3, 1] and x.tolist() == [1, 2, 3]
    coo = L.new_COO_matrix(B)
    c = coo.contents
    assert np.ctypeslib.as_array(c.rows, shape=(3,)).tolist() == [0, 0, 2]
    L.free_COO_matrix(coo)
    # lower-triangular COO + refresh (upstream src/sparse/COO_matrix.c:48-98)
    H = HostCSR([0, 2, 4, 5], [0, 1, 0, 1, 2], [1., 2., 2., 3., 4.], 3, 3)
    lt = L.new_COO_matrix_lower_triangular(H.ref)
    c = lt.contents
    assert c.nnz == 4
    assert np.ctypeslib.as_array(c.value_map, shape=(4,)).tolist() == [0, 2, 3, 4]
    vals = np.array([10., 20., 30., 40., 50.])
    L.refresh_lower_triangular_coo(lt, vals.ctypes.data)
    assert np.ctypeslib.as_array(c.x, shape=(4,)).tolist() == [10., 30., 40., 50.]
    L.free_COO_matrix(lt)
    L.free_CSR_matrix(A)
    L.free_CSR_matrix(B)


@pytest.mark.skipif(GPU, reason="checks the no-device behaviour")
def test_no_device_fails_loudly_status_mode():
    L = _lib.lib()
    assert L.sdl_device_available() == 0
    L.sdl_set_fatal_errors(0)
    try:
        H = HostCSR([0, 1], [0], [1.0], 1, 1)
        iw = np.zeros(1, np.int32)
        out = L.csr_to_csc_alloc(H.ref, iw.ctypes.data_as(C.POINTER(C.c_int)))
        assert not out, "must not compute without a device"
        assert L.sdl_last_status() == 1  # SDL_ERR_NO_DEVICE
        assert b"no CUDA device" in L.sdl_last_error()
    finally:
        L.sdl_set_fatal_errors(1)


@pytest.mark.skipif(GPU, reason="checks the no-device behaviour")
def test_no_device_fatal_mode_exits():
    code = (
        "import ctypes as C, numpy as np, sys\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "from sparsediff_linalg_b200 import _lib\n"
        "from sparsediff_linalg_b200.host import HostCSR\n"
        "L = _lib.lib()\n"
        "H = HostCSR([0, 1], [0], [1.0], 1, 1)\n"
        "L.transpose(H.ref, None)\n"
        "print('unreachable')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "unreachable" not in r.stdout
    assert "no CUDA device" in r.stderr
