"""Build libfeti4i_b200.so in-tree: host C++ (OpenMP) + CUDA for sm_100a.

    python -m espreso_b200.build          # incremental
    python -m espreso_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfeti4i_b200.so")
# the same library with the FETI4I_INT_WIDTH 64 ABI (FETI4IInt = long)
LIB64 = os.path.join(HERE, "libfeti4i_b200_i64.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = "-fPIC,-fopenmp,-march=x86-64-v3,-O3,-Wall,-Wno-unused-function"
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", HOST_FLAGS, "-I", os.path.join(ROOT, "include")]

SOURCES = ["dense.cpp", "decompose.cpp", "prep.cpp", "hybrid.cpp", "feti4i.cpp", "gpu_solver.cu", "gpu_prep.cu"]
HEADERS = ["common.h", "dense.h", "decompose.h", "prep.h", "gpu_solver.h", "gpu_prep.h", "hybrid.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h)
                                                      for h in ("feti4i.h", "feti4i_ext.h", "mpi.h")]
    objs = []
    units = [(src, os.path.splitext(src)[0] + ".o", []) for src in SOURCES]
    units.append(("feti4i.cpp", "feti4i_i64.o", ["-DFETI4I_INT_WIDTH=64"]))
    for src, obj, defs in units:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, obj)
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + COMMON + defs + ARCH + ["-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"compilation of {src} failed:\n{r.stdout}\n{r.stderr}")
            if verbose and r.stderr:
                print(r.stderr)
    shared = [o for o in objs if not os.path.basename(o).startswith("feti4i")]
    abi32 = os.path.join(BUILD, "feti4i.o")
    abi64 = os.path.join(BUILD, "feti4i_i64.o")
    for lib, abi in ((LIB, abi32), (LIB64, abi64)):
        if force or _newer(lib, shared + [abi]):
            cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-o", lib] + shared + [abi, "-lgomp"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
