"""Compile ``csrc/pyib_b200.cu`` into the in-tree ``libpyib_b200.so`` for sm_100a.

``--fmad=false`` keeps every scalar expression rounded like the NumPy
reference (no contracted multiply-adds), which the bit-exact stencil and
spreading parity relies on.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc" / "pyib_b200.cu"
OUT = HERE / "libpyib_b200.so"
INCLUDE = HERE.parent / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the B200 library cannot be built")
    return cand


def build_library(force=False, verbose=False):
    """Build libpyib_b200.so if it is missing or older than its sources."""
    deps = [SRC, INCLUDE / "pyib_b200.h"]
    if OUT.exists() and not force and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-o", str(OUT) + ".tmp", str(SRC)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(str(OUT) + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build_library(force=True, verbose=True)
