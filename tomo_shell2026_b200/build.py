"""Build libtomo_b200.so in-tree (nvcc, sm_100a only).

The library is compiled straight from tomo_shell2026_b200/csrc/*.cu with
``-gencode arch=compute_100a,code=sm_100a``.  Device code uses explicit
round-to-nearest intrinsics and ``-fmad=false`` so no multiply-add is ever
contracted; host code (rotation matrices, mass model) is compiled with
``-ffp-contract=off`` and without fast-math, like the reference engine.
The result lands in tomo_shell2026_b200/_lib/ so it travels with the tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libtomo_b200.so"
INCLUDE = PKG.parent / "include"
NVCC = os.environ.get("NVCC", str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"))

SOURCES = ["tomo_kernels.cu", "tomo_engine.cu", "tomo_mlp.cu"]
HEADERS = ["tomo_common.cuh", "tomo_mlp.cuh", "tomo_span.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fno-fast-math",
    "--shared",
]


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [INCLUDE / "tomo_b200.h", Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    """Compile the CUDA library if any source is newer than it."""
    if not force and not _stale():
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose_ptxas else []),
           *[str(CSRC / s) for s in SOURCES], "-o", str(tmp)]
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + proc.stdout[-6000:])
    if verbose_ptxas:
        print(proc.stdout)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="force" in sys.argv, verbose_ptxas="-v" in sys.argv))
