"""Build the sm_100a shared library of the step: vlasolve_b200/libvlasolve_b200.so.

nvcc compiles the CUDA kernels and the C++ host code (C-ABI, set-up) into one
in-tree shared object, with explicit -gencode for sm_100a (no PTX fallback
for other architectures).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvlasolve_b200.so")
DRIVER = os.path.join(HERE, "vlasolve_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["vls_kernels.cu", "vls_rc.cu", "vls_adjoint.cu", "vls_noalloc.cu", "vls_spline.cu",
           "vls_profile.cu",
           "vls_api.cpp",
           "vls_setup.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp",
          "-I" + os.path.join(REPO, "include")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(REPO, "include", "vlasolve_b200.h"))
    deps.append(os.path.join(REPO, "include", "vlasolve_b200.hpp"))
    deps.append(os.path.join(CSRC, "vls_main.cpp"))
    if not force and not _stale(LIB, deps) and os.path.exists(DRIVER):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s + ".o")
        cmd = [NVCC, "-c", src, "-o", obj] + ARCH + COMMON
        if s.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "cu"] if False else []
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fopenmp",
                                                          "-lgomp", "-lcudart"]
    subprocess.check_call(cmd)
    # command-line driver with the reference's options (links the library)
    subprocess.check_call([
        "g++", "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"),
        os.path.join(CSRC, "vls_main.cpp"), "-L" + HERE, "-lvlasolve_b200",
        "-Wl,-rpath,$ORIGIN", "-o", DRIVER])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
