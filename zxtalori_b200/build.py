"""Build the engine's shared library in-tree: zxtalori_b200/_lib/libzxtalori.so.

nvcc compiles every source for sm_100a (Blackwell B200) with line info, links the CUDA
runtime statically, and exports only the C ABI declared in include/zxtalori.h. No GPU is
needed to build.

    python -m zxtalori_b200.build            # or: python zxtalori_b200/build.py
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SRC = HERE / "csrc"
OUT = HERE / "_lib"
LIB = OUT / "libzxtalori.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["kernels.cu", "engine.cpp", "groups.cpp", "hopf.cpp", "exports.cpp", "memory.cpp", "no_alloc.cu", "batch.cpp", "cover.cpp", "insert.cpp", "optimize.cpp", "serve.cpp"]


def nvcc():
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found")


def _flags():
    return ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   "-I", str(SRC), "-I", str(ROOT / "include")]


def _compile(source, objdir):
    src = SRC / source
    obj = objdir / (source + ".o")
    lang = [] if source.endswith(".cu") else ["-x", "cu"]
    cmd = [nvcc()] + _flags() + lang + ["-c", str(src), "-o", str(obj)]
    subprocess.run(cmd, check=True)
    return obj


def stale():
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    inputs = list(SRC.glob("*")) + [ROOT / "include" / "zxtalori.h", Path(__file__)]
    return any(p.stat().st_mtime > built for p in inputs if p.is_file())


def build(force=False, verbose=True):
    if not force and not stale():
        return LIB
    OUT.mkdir(exist_ok=True)
    objdir = OUT / "obj"
    objdir.mkdir(exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objects = list(pool.map(lambda s: _compile(s, objdir), SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objects]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
