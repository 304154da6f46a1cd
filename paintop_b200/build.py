"""Build ``libpaintop_cuda.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m paintop_b200.build [--verbose]`` (``--verbose`` adds
``-Xptxas -v`` to print registers, spills and shared memory per kernel).
Objects go to ``paintop_b200/_build/``; the library lands next to this file so
it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpaintop_cuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                   "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
SOURCES = ["rbsor_kernels.cu", "solver_host.cu", "op_host.cpp", "autotune.cpp", "noalloc.cu",
           "mask_kernels.cu", "mg_solver.cu", "unet/unet_kernels.cu", "unet/conv_tma.cu", "unet/unet.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(d, f) for d in (CSRC, os.path.join(CSRC, "unet")) for f in os.listdir(d)
               if f.endswith((".h", ".cuh", ".inc"))]
    headers.append(os.path.join(ROOT, "include", "paintop_cuda.h"))
    objs = []
    changed = force
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src.replace("/", "_") + ".o")
        objs.append(obj)
        if force or verbose or _stale(obj, [path] + headers):
            cmd = [nvcc()] + CU_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd[1:1] = ["-x", "cu"]
            subprocess.run(cmd, check=True)
            changed = True
    if changed or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt",
                                                                          "-ldl", "-lpthread"],
                       check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
