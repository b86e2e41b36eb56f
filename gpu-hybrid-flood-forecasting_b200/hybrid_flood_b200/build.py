"""Compile the sm_100a CUDA library ``lib/libswe_b200.so`` in-tree with nvcc.

    python -m hybrid_flood_b200.build [--force] [--verbose]

The library is a plain C-ABI shared object (``include/swe_b200.h``); it links
the CUDA runtime statically and has no PyTorch dependency, so the same file is
usable from ctypes, cgo, JNI or a C/C++ host.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent                      # gpu-hybrid-flood-forecasting_b200/
REPO = ROOT.parent
CSRC = ROOT / "csrc"
INCLUDE = REPO / "include"
LIB = PKG / "lib" / "libswe_b200.so"
SOURCES = [CSRC / "swe_api.cu"]
DEPS = SOURCES + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libswe_b200.so")


def is_stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    return any(p.stat().st_mtime > built for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Build the library if missing or older than its sources; return its path."""
    if not force and not is_stale():
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC,-O2", "-shared", "-I", str(INCLUDE),
        *(["-Xptxas", "-v"] if verbose else []),
        *map(str, SOURCES), "-o", str(tmp),
    ]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
