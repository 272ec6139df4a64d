"""Builds the sm_100a shared library libsf2d_b200.so in-tree with nvcc.

    python -m specfem2d_b200.build

The library is the product's C ABI (include/sf2d_b200.h); it links only the
CUDA runtime.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libsf2d_b200.so")
SOURCES = ["sf2d_elastic.cu", "sf2d_fwi.cu", "sf2d_noalloc.cu", "sf2d_coupled.cu", "sf2d_tiler.cpp",
           "sf2d_fortran.cpp", "sf2d_smooth.cu", "sf2d_batch.cu"]
HEADERS = ["sf2d_tiler.h", "sf2d_kernels.cuh", "sf2d_runtime.h", "sf2d_acoustic.cuh", "sf2d_pml.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
OBJDIR = os.path.join(PKG, "_build")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def export_map() -> str:
    """Linker version script: the library exports its C ABI (sf2d_*) and the
    reference's Fortran entry points (include/sf2d_fortran.h) and nothing else,
    so that none of its C++ internals can bind to a host's symbols."""
    with open(os.path.join(ROOT, "include", "sf2d_fortran.h")) as f:
        names = sorted(set(re.findall(r"^void (\w+_)\(", f.read(), re.M)))
    return "{\n  global:\n    sf2d_*;\n" + "".join(f"    {n};\n" for n in names) + "  local:\n    *;\n};\n"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [
        os.path.join(ROOT, "include", h) for h in ("sf2d_b200.h", "sf2d_coupled.h", "sf2d_fortran.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in parallel, then links the shared
    library against the static CUDA runtime."""
    from concurrent.futures import ThreadPoolExecutor

    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    cmds = [[NVCC, *FLAGS, "-c", os.path.join(CSRC, s), "-o", o] for s, o in zip(SOURCES, objs)]

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd).returncode

    with ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        codes = list(ex.map(compile_one, cmds))
    if any(codes):
        raise subprocess.CalledProcessError(max(codes), "nvcc")
    mapfile = os.path.join(OBJDIR, "libsf2d_b200.map")
    with open(mapfile, "w") as f:
        f.write(export_map())
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static", *objs,
            "-Xlinker", "--version-script=" + mapfile, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
