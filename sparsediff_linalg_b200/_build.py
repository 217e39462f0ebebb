"""Build recipe for the in-tree CUDA library ``libsparsediff_linalg_b200.so``.

Every ``csrc/*.cu`` / ``csrc/*.cpp`` is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) into ``_build/`` and linked into one
shared library next to this file. ``--fmad=false`` keeps nvcc from contracting any
multiply-add into an FMA, so the FP64 roundings are the ones the sources spell out.
Objects are rebuilt only when their source or a header under ``csrc/`` / ``include/``
is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB_NAME = "libsparsediff_linalg_b200.so"
LIB_PATH = PKG / LIB_NAME

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-O3,-Wall", "-I", str(INCLUDE), "-I", str(CSRC),
]


def _nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(home) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found (set CUDA_HOME)")
    return found


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.rglob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, hdr_mtime: float, extra: list[str]) -> str | None:
    if obj.exists():
        om = obj.stat().st_mtime
        if om >= src.stat().st_mtime and om >= hdr_mtime:
            return None
    cmd = [_nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return src.name


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile every source and link the library. Returns the library path."""
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    hdr = _headers_mtime()
    extra = list(extra_flags or [])
    objs = [BUILD / (s.name + ".o") for s in srcs]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        futs = [ex.submit(_compile, s, o, hdr, extra) for s, o in zip(srcs, objs)]
        rebuilt = [f.result() for f in futs]
    rebuilt = [r for r in rebuilt if r]
    if rebuilt or not LIB_PATH.exists() or any(o.stat().st_mtime > LIB_PATH.stat().st_mtime for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB_PATH), *map(str, objs),
               "-Xlinker", "-Bsymbolic", "-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB_PATH} (recompiled: {', '.join(rebuilt) or 'nothing'})")
    return LIB_PATH


if __name__ == "__main__":
    build(verbose=True, extra_flags=sys.argv[1:])
