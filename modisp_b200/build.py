"""Compile the engine library in-tree for sm_100a.

    python -m modisp_b200.build        # -> modisp_b200/_lib/libmodisp_b200.so

The library is a plain shared object exporting the C ABI of
``include/modisp_b200.h``; the Python package binds it with ctypes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "_lib"
LIBRARY = LIBDIR / "libmodisp_b200.so"
SOURCES = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "modisp_b200.h"]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; the modisp_b200 engine needs the CUDA 12.9 toolkit to build")


def command(output: Path = LIBRARY, verbose_ptxas: bool = False) -> list[str]:
    # single-precision division and square root as hardware approximations, and
    # FP32 denormals flushed: the FP32 scan only decides signs (FP64 is untouched)
    cmd = [nvcc(), ARCH, "-lineinfo", "-O3", "-std=c++17", "-prec-div=false", "-prec-sqrt=false", "-ftz=true",
           "-Xcompiler", "-fPIC", "-shared",
           f"-I{ROOT / 'include'}", str(CSRC / "engine.cu"), "-o", str(output)]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def up_to_date() -> bool:
    if not LIBRARY.exists():
        return False
    built = LIBRARY.stat().st_mtime
    return all(src.stat().st_mtime <= built for src in SOURCES if src.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    tmp = LIBRARY.with_suffix(".so.tmp")
    result = subprocess.run(command(tmp, verbose), capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + result.stdout + result.stderr)
    if verbose:
        sys.stderr.write(result.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(path)
