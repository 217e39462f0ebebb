"""B200-native sparse-product path of sparsediff_linalg.

The product is the CUDA library ``libsparsediff_linalg_b200.so`` built in this
directory; it exports the upstream C API (``include/sparsediff_linalg/*.h``) and the
device-resident extension (``include/sparsediff_linalg_cuda.h``). This package is a
thin ctypes layer over that library:

* ``lib()``: the loaded library with every C signature bound;
* ``host``: numpy <-> C struct helpers for the upstream host-pointer API;
* ``device``: torch-tensor wrappers of the device-resident API;
* ``workloads``: seeded synthetic inputs of the benchmark configurations.
"""
from ._lib import SDLError, check, lib, LIB_PATH  # noqa: F401

__all__ = ["lib", "check", "SDLError", "LIB_PATH"]
