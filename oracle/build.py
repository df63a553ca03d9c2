"""Build recipes for the parity oracles (test infrastructure only).

Two libraries come out of here:

* ``oracle/_build/libtomo_oracle.so`` -- the plain-C restatement of the
  reference INT3 orientation-search path (``oracle/tomo_oracle.c``).
* ``oracle/_ref/libtomo_ref.so`` -- the reference INT3 engine itself, compiled
  from its own sources where they lie under the reference checkout
  (``cfms_tomo/Tomo_Shell_vc_src``) plus the thin driver in
  ``oracle/ref/ref_driver.cpp``.  Only this recipe reads the reference tree;
  the built ``.so`` is what travels to GPU hosts.  When the reference checkout
  is absent the recipe is skipped and an already-built library is used.

Both are compiled with ``-O2 -ffp-contract=off`` and without ``-march`` /
``-ffast-math`` so that x86-64 SSE single-precision semantics hold exactly.
The product library never links or loads either of them.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ORACLE_DIR = Path(__file__).resolve().parent
BUILD_DIR = ORACLE_DIR / "_build"
REF_OUT = ORACLE_DIR / "_ref"
# The reference checkout: TOMO_REFERENCE_ROOT when set, else a directory named
# "reference" beside this repository's root.
REF_ROOT = Path(os.environ.get("TOMO_REFERENCE_ROOT", str(ORACLE_DIR.parent.parent / "reference")))
REF_SRC = REF_ROOT / "cfms_tomo" / "Tomo_Shell_vc_src"
CUDA_INC = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"

ORACLE_LIB = BUILD_DIR / "libtomo_oracle.so"
REF_LIB = REF_OUT / "libtomo_ref.so"

# Reference translation units on the INT3 path (and what they drag in through
# STomoSh_Base / S3DPrinterInfo).  Tomo_Shell2026.cpp is not built: it also
# hosts the CUDA engine; its orchestration is mirrored by ref_driver.cpp.
REF_UNITS = [
    "Tomo_types.cpp",
    "cpu_src/STomoSh_INT3.cpp",
    "cpu_src/STomoSh_Base.cpp",
    "cpu_src/STomoVoxelSpaceInfo.cpp",
    "cpu_src/S3DPrinterInfo.cpp",
    "cpu_src/STomoVolMassInfo.cpp",
    "cpu_src/SMatrix4f.cpp",
    "cpu_src/STomoAABB3Df.cpp",
    "cpu_src/STomoAABB2D.cpp",
    "cpu_src/STPSlot.cpp",
    "cpu_src/STomoPixel.cpp",
    "cpu_src/STomoVoxel.cpp",
    "cpu_src/STomoTriangle.cpp",
    "cuda_src/SYPRInfo.cpp",
]

KEEP_INLINE_EXEMPT = {"S3DPrinterInfo.cpp", "SYPRInfo.cpp", "cuda_host_stubs.cpp"}

COMMON_FLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-g0"]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + proc.stdout[-4000:])


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.exists() and s.stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    """Compile the C restatement into oracle/_build/libtomo_oracle.so."""
    src = ORACLE_DIR / "tomo_oracle.c"
    hdr = ORACLE_DIR / "tomo_oracle.h"
    BUILD_DIR.mkdir(exist_ok=True)
    if force or _stale(ORACLE_LIB, [src, hdr, Path(__file__)]):
        tmp = ORACLE_LIB.with_suffix(".so.tmp")
        _run(["gcc", "-std=c11", *COMMON_FLAGS, "-Wall", "-Wextra", "-pthread", "-shared",
              str(src), "-o", str(tmp), "-lm"])
        tmp.replace(ORACLE_LIB)
    return ORACLE_LIB


def _write_forwarders(gen: Path) -> None:
    """The reference headers include "..\\Tomo_types.h" with a Windows path
    separator (cpu_src/S3DPrinterInfo.h:2, STomoAABB2D.h:2, STomoAABB3Df.h:2,
    STomoVolMassInfo.h:2, cuda_src/CUDA_types.cuh:9).  On Linux that is a
    single file name containing a backslash, so a one-line forwarding header
    with that literal name is placed on the include path."""
    gen.mkdir(parents=True, exist_ok=True)
    fwd = gen / "..\\Tomo_types.h"
    text = f'#include "{REF_SRC / "Tomo_types.h"}"\n'
    if not fwd.exists() or fwd.read_text() != text:
        fwd.write_text(text)


def reference_available() -> bool:
    return (REF_SRC / "cpu_src" / "STomoSh_INT3.cpp").exists()


def build_ref(force: bool = False) -> Path | None:
    """Compile the reference INT3 engine from its own sources into
    oracle/_ref/libtomo_ref.so.  Returns None when neither the reference
    checkout nor a prebuilt library is present."""
    if not reference_available():
        return REF_LIB if REF_LIB.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    objdir = REF_OUT / "obj"
    objdir.mkdir(exist_ok=True)
    gen = REF_OUT / "shim_gen"
    _write_forwarders(gen)
    incs = ["-I", str(gen), "-I", str(ORACLE_DIR / "ref" / "shim"), "-I", str(REF_SRC),
            "-I", str(CUDA_INC)]
    cxx = ["g++", "-std=c++17", *COMMON_FLAGS, "-w", "-pthread"]
    objs: list[Path] = []
    own = [ORACLE_DIR / "ref" / "ref_driver.cpp", ORACLE_DIR / "ref" / "cuda_host_stubs.cpp"]
    shim = ORACLE_DIR / "ref" / "shim" / "windows.h"
    for unit in REF_UNITS + [str(p) for p in own]:
        src = Path(unit) if os.path.isabs(unit) else REF_SRC / unit
        obj = objdir / (src.stem + ".o")
        # MSVC-style inline definitions in .cpp files (Tomo_types.cpp:14-159,
        # STomoPixel.cpp) are used from other units; keep them out of line.
        # Units that include the CUDA runtime headers must not, or every
        # header inline would pull a libcudart symbol into the oracle.
        keep = [] if src.name in KEEP_INLINE_EXEMPT else ["-fkeep-inline-functions"]
        if force or _stale(obj, [src, shim, Path(__file__)]):
            _run([*cxx, *keep, *incs, "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    if force or _stale(REF_LIB, objs):
        tmp = REF_LIB.with_suffix(".so.tmp")
        _run(["g++", "-shared", "-pthread", "-Wl,--no-undefined", *map(str, objs), "-o", str(tmp), "-lm"])
        tmp.replace(REF_LIB)
    return REF_LIB


def clean() -> None:
    for d in (BUILD_DIR, REF_OUT):
        if d.exists():
            shutil.rmtree(d)


if __name__ == "__main__":
    what = sys.argv[1:] or ["oracle", "ref"]
    if "clean" in what:
        clean()
    if "oracle" in what:
        print(build_oracle(force="force" in what))
    if "ref" in what:
        print(build_ref(force="force" in what))
