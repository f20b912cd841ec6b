"""Build libaed.so in place: nvcc for sm_100a, g++ for the host C++.

    python -m alps_b200.build [--force]

Objects go to alps_b200/_build/ (git-ignored); the library lands at
alps_b200/libaed.so so that it travels with the source tree.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaed.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
             "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["kernels.cu", "noalloc.cu", "batch.cu", "momentum.cu", "measure.cu", "spin.cu", "refine.cu"]
CPP_SOURCES = ["model.cpp", "tmatrix.cpp", "api.cpp", "lanczos.cpp", "server.cpp"]
HEADERS = ["aed_internal.h", "rr_core.h", "kernels.cuh", "handle.h", "reduce.cuh", "apply.cuh", "apply_blocks.cuh", "apply_stream.cuh",
           "tmatrix_core.h",
           "batch.cuh", "momentum.cuh", "spin.cuh"]


def _newer(src, dst, deps):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "aed.h")]
    objs = []
    cmds = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer(src, obj, deps):
            cmds.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _newer(src, obj, deps):
            cmds.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c))
        procs.append((c, subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    errs = []
    for c, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append(" ".join(c) + "\n" + out.decode())
        elif verbose and out:
            print(out.decode())
    if errs:
        raise RuntimeError("libaed build failed:\n" + "\n".join(errs))
    if force or cmds or not os.path.exists(LIB):
        link = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(link))
        subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
