"""In-tree build of the native library for sm_100a.

``python -m snusolver_b200.build`` compiles the host C++ (structure, front
plan, C-ABI), the CUDA engine (nvcc, ``-gencode arch=compute_100a,
code=sm_100a``) and links ``snusolver_b200/libsnusolver_b200.so`` with the
CUDA runtime and METIS linked statically, plus the ``driver`` command-line
program next to it.  Objects go to ``snusolver_b200/_build``; unchanged
sources are not recompiled.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
METIS = os.path.join(CUDA, "targets", "x86_64-linux", "lib", "libmetis_static.a")
LIB = os.path.join(HERE, "libsnusolver_b200.so")
DRIVER = os.path.join(HERE, "driver")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
            f"-I{CUDA}/include", f"-I{ROOT}/include"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", f"-I{ROOT}/include"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
               + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
               + glob.glob(os.path.join(ROOT, "include", "*.h")))
    objs = []
    lib_srcs = [s for s in glob.glob(os.path.join(CSRC, "**", "*.cpp"),
                                     recursive=True)
                if not s.endswith("driver.cpp")]
    for src in sorted(lib_srcs):
        obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace("/", "_") + ".o")
        if _stale(obj, [src] + headers):
            _run(["g++"] + CXXFLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "**", "*.cu"), recursive=True)):
        obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace("/", "_") + ".o")
        if _stale(obj, [src] + headers):
            _run([NVCC] + NVFLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
             + [METIS, "-Xlinker", "--exclude-libs,ALL", "-lpthread", "-ldl",
                "-lrt"], verbose)
    drv = os.path.join(CSRC, "driver.cpp")
    if os.path.exists(drv) and _stale(DRIVER, [drv, LIB] + headers):
        _run(["g++"] + CXXFLAGS + [drv, "-o", DRIVER, f"-L{HERE}",
                                   "-lsnusolver_b200", "-Wl,-rpath,$ORIGIN"],
             verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
