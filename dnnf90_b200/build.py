"""Build of the device library libdnnf90_b200.so (nvcc, sm_100a only).

The library is built in-tree into dnnf90_b200/_lib so that it travels with
the repository; ``python -m dnnf90_b200.build`` or ``build()``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libdnnf90_b200.so")

SOURCES = ["tables.cpp", "bell_plan.cpp", "tile_plan.cpp", "api.cpp", "engine.cu", "bell.cu",
           "bell_tile.cu", "gemm_tc.cu", "gemm_f64.cu", "ngd.cu", "kalman.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-Xcompiler", "-Wall"]


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(src: str, obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def build(verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    headers += [os.path.join(HERE, "..", "include", f)
                for f in os.listdir(os.path.join(HERE, "..", "include"))]
    objs = []
    changed = False
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if not _stale(src, obj, headers):
            continue
        cmd = [nvcc] + ARCH + NVFLAGS + ["-c", src, "-o", obj]
        if s.endswith(".cpp"):
            cmd = [nvcc] + NVFLAGS + ["-x", "cu"] + ARCH + ["-c", src, "-o", obj]
        if ptxas_v and s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        changed = True
    if changed or not os.path.exists(LIB):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
