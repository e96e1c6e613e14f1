"""Build recipe for libhdgrid.so (sm_100a) and the search-engine binary.

Compiles every source under hdgrid_b200/csrc with nvcc into an in-tree shared library,
so the built artefact travels with the source tree.  Usage: python hdgrid_b200/build_native.py
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libhdgrid.so"
BIN = PKG / "bin" / "search-engine"
BUILD = PKG / "_build"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr"]

LIB_SOURCES = [
    "hdg_config.cpp",
    "hdg_abi.cpp",
    "hdg_io.cpp",
    "hdg_build.cu",
    "hdg_query.cu",
    "hdg_kernels_ref.cu",
    "hdg_gemm.cu",
    "hdg_learned.cu",
]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "hdgrid.h"]
    objs = []
    for src in LIB_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        extra = ["-Xptxas", "-v"] if (verbose_ptxas and s.suffix == ".cu") else []
        lang = ["-x", "cu"] if s.suffix == ".cu" else ["-x", "c++"]
        _run([NVCC, *ARCH, *COMMON, *extra, *lang, "-c", str(s), "-o", str(o)])
    if force or not _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(LIB), *map(str, objs), "-lcudart"])
    main = CSRC / "search_engine_main.cpp"
    if main.exists():
        BIN.parent.mkdir(exist_ok=True)
        if force or not _newer(BIN, [main, LIB] + headers):
            _run([NVCC, *ARCH, "-O2", "-std=c++17", "-x", "c++", str(main), "-o", str(BIN),
                  "-L" + str(PKG), "-lhdgrid", "-Xlinker", "-rpath,$ORIGIN/..", "-lcudart"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
