"""Build recipe of libhp2d.so (sm_100a), in-tree next to this file.

    python -m hydropol2d_b200.build

nvcc cross-compiles without a GPU.  -fmad=false keeps every multiply and add separately
rounded so the kernels reproduce the CPU restatement bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
LIB = PKG / "libhp2d.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC",
]
# No --split-compile: with it the device code of a kernel depended on how nvcc partitioned the
# translation unit among the build machine's threads, and two builds of the same source ran the
# 2048^2 Green-Ampt + rain-map step at 15 or 19 GCUPS and the wet step at 39 or 37; whole-unit
# builds run at 21 and 39 every time.
SPLIT: list[str] = []


def sources() -> list[Path]:
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cuh")) + [ROOT / "include" / "hp2d.h"]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources())


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every csrc/*.cu to an object in parallel (the build folder is PKG/_build),
    then links libhp2d.so."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    out_dir = PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    inc = [f"-I{ROOT / 'include'}", f"-I{SRC}"]
    cus = sorted(SRC.glob("*.cu"))

    def compile_one(cu: Path) -> Path:
        obj = out_dir / (cu.stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, *SPLIT, *inc, "-c", str(cu), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(cus)) as ex:
        objs = list(ex.map(compile_one, cus))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *[str(o) for o in objs],
           "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
