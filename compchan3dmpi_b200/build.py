"""In-tree build of the CUDA library for sm_100a.

    python -m compchan3dmpi_b200.build [--force]

Produces ``compchan3dmpi_b200/lib/libchanrhs.so`` with nvcc directly (no JIT
cache), so the built file travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SRC = HERE / "csrc"
OUT = HERE / "lib" / "libchanrhs.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread", "-shared",
         f"-I{ROOT / 'include'}"]


def sources():
    return [SRC / "chanrhs.cu", SRC / "closure.cu", SRC / "deck_io.cpp"]


def deps():
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cuh")) + sorted(SRC.glob("*.cpp")) + \
        [ROOT / "include" / "chanrhs.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if not force and OUT.exists():
        newest = max(p.stat().st_mtime for p in deps())
        if OUT.stat().st_mtime >= newest:
            return OUT
    tmp = OUT.with_suffix(f".{os.getpid()}.tmp.so")
    cmd = [NVCC, *ARCH, *FLAGS, "-o", str(tmp), *map(str, sources())]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
