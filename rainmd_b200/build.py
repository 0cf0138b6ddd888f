"""Compile the engine's CUDA sources into rainmd_b200/librmd.so for sm_100a.

The library is a plain shared object with a C ABI (include/rmd.h); it is built in-tree
with nvcc and loaded by ctypes (rainmd_b200/_lib.py) or by a Node N-API addon.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "librmd.so")
SOURCES = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
HEADERS = sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
                 + [os.path.join(os.path.dirname(HERE), "include", "rmd.h")])
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > built for p in SOURCES + HEADERS)


# Sources whose floating-point results must not depend on the compiler's choice of fused
# multiply-adds (the renderer: its image is compared bit for bit with a CPU restatement).
UNFUSED = {"raster.cu"}
OBJ_DIR = os.path.join(os.path.dirname(HERE), "_build")


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    extra = ["-Xptxas", "-v"] if verbose else []
    fused = [s for s in SOURCES if os.path.basename(s) not in UNFUSED]
    objects = []
    os.makedirs(OBJ_DIR, exist_ok=True)
    for src in SOURCES:
        if os.path.basename(src) not in UNFUSED:
            continue
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        flags = [f for f in FLAGS if f != "-shared"]
        cmd = [NVCC, *flags, *extra, "-fmad=false", "-c", "-o", obj, src]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            sys.stderr.write(result.stdout + result.stderr)
            raise RuntimeError(f"nvcc failed to compile {os.path.basename(src)}")
        if verbose:
            sys.stderr.write(result.stderr)
        objects.append(obj)
    cmd = [NVCC, *FLAGS, *extra, "-o", LIB, *fused, *objects]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("nvcc failed to build librmd.so")
    if verbose:
        sys.stderr.write(result.stderr)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)
