"""Build recipe for libtomo_b200.so (in-tree, sm_100a).

Compiles every CUDA source with nvcc for ``-gencode arch=compute_100a,code=sm_100a`` and the
host C++ sources with g++, then links one shared library into
``seismic_tomography_3d_b200/_lib/``.  Incremental: objects are rebuilt only when a source
or header is newer.  Usable as ``python -m seismic_tomography_3d_b200.build``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libtomo_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
# Sources that restate a reference FP32 computation bit for bit: no FMA contraction.
NO_FMA_SOURCES = {"fsm.cu"}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
             "-I" + os.path.join(CUDA, "include"), "-I" + os.path.join(ROOT, "include")]


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            if os.path.basename(src) in NO_FMA_SOURCES:
                extra += ["-fmad=false"]
            _run([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj], verbose)
    host_hdrs = hdrs + glob.glob(os.path.join(HOST, "*.hpp"))
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp")) + glob.glob(os.path.join(HOST, "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + host_hdrs):
            _run([CXX] + CXX_FLAGS + ["-c", src, "-o", obj], verbose)
    if _stale(LIB, objs):
        # -Bsymbolic: calls inside the library bind to its own definitions even when another
        # library in the process exports the same C++ names (e.g. the reference's own
        # catch_parameter when both are loaded for a parity test)
        _run([NVCC] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", LIB] + objs
             + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"], verbose)
    # drop-in executables (the reference's eikonal.exe / tomography.exe flows)
    for src in sorted(glob.glob(os.path.join(HOST, "apps", "*_main.cpp"))):
        exe = os.path.join(LIBDIR, os.path.basename(src)[:-len("_main.cpp")])
        if _stale(exe, [src, LIB] + host_hdrs):
            _run([CXX] + CXX_FLAGS + [src, "-o", exe, "-L" + LIBDIR, "-ltomo_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
