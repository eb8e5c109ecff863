"""Build the in-tree CUDA library (sm_100a) with nvcc.

Produces cfdsfemmpi_b200/libcfdgpu.so from csrc/*.cu and csrc/*.cpp.  The
library links only the CUDA runtime; the Python layer loads it with ctypes.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcfdgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2",
              "-Xptxas", "-O3"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources() + headers())


HOST = os.path.join(HERE, "host")
BIN = os.path.join(HERE, "bin")
PROGRAMS = {"cfdsfemmpi": "cfdsfemmpi.cpp", "test-ldc-stru": "test-ldc-stru.cpp"}


def build_host(verbose: bool = False) -> None:
    """The C++ driver (StabFEM) and the reference-shaped command-line programs."""
    os.makedirs(BIN, exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include")
    cuda_lib = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64")
    deps = [os.path.join(HOST, f) for f in os.listdir(HOST)] + [LIB]
    for prog, main in PROGRAMS.items():
        out = os.path.join(BIN, prog)
        if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-I", inc, "-o", out, os.path.join(HOST, main),
               os.path.join(HOST, "StabFEM.cpp"), "-L", HERE, "-lcfdgpu", "-L", cuda_lib, "-lcudart",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        build_host(verbose)
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp", *sources(), "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    build_host(verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
