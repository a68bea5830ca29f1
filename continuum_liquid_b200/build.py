"""Builds libclb200.so in-tree with nvcc for sm_100a (B200).

The library is one translation unit (csrc/clb200.cu). It is compiled with -fmad=false so that every
floating-point operation is separately rounded, which the bit-exact parity of the solver kernels
relies on.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR / "csrc"
LIBRARY = PACKAGE_DIR / "libclb200.so"
SOURCES = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh"))
HEADERS = [PACKAGE_DIR.parent / "include" / "clb200.h"]

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-fmad=false",
    "-Xcompiler",
    "-fPIC",
    "-shared",
]


def nvcc_path() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libclb200.so")


def is_stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(path.stat().st_mtime > built for path in [*SOURCES, *HEADERS] if path.exists())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile csrc/clb200.cu into libclb200.so next to this file (skipped when up to date)."""
    if not force and not is_stale():
        return LIBRARY
    command = [nvcc_path(), *NVCC_FLAGS, "-o", str(LIBRARY), str(CSRC / "clb200.cu")]
    if verbose:
        print(" ".join(command))
    result = subprocess.run(command, cwd=CSRC, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed ({result.returncode}):\n{result.stdout}\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
