"""Build libxr.so in place (sm_100a only).

    python xray-directional-reconstruction_b200/build.py [--force]

CUDA sources: nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3.
Host C++ (xr_host.cpp): g++ -O2 -ffp-contract=off without -march flags, so
the per-view geometry tables round exactly like the reference's FP32 code.
The CUDA runtime is linked statically, so the library loads without
LD_LIBRARY_PATH.  Objects go to _build/ beside this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxr.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["xr_kernels.cu", "xr_column.cu", "xr_orient.cu", "xr_fdk.cu", "xr_static.cu", "xr_learn.cu", "xr_solver.cu",
              "xr_fiber.cu"]
CXX_SOURCES = ["xr_host.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "xr.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-Xptxas", "-v" if verbose else "-O3", "-c", s, "-o", o]
            r = _run(cmd)
            if verbose:
                sys.stdout.write(r.stderr)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cxx = shutil.which("g++") or "g++"
            _run([cxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                  "-I", os.path.join(CUDA, "include"), "-c", s, "-o", o])
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
