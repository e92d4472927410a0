"""Builds thor_b200/libthorx.so (the CUDA kernels and the C ABI) for sm_100a with nvcc.

    python -m thor_b200.build          # or build() from __graft_entry__.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libthorx.so")

SOURCES = ["thorx_capi.cu", "dyn_fp64.cu", "rt.cu", "globdiag.cu", "surrogate.cu", "icogrid.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-fopenmp", "-shared", "-lgomp",
              "-I" + os.path.join(ROOT, "include")]
# the environment's default host compiler may lack the OpenMP runtime; the system g++ has it
if os.path.exists("/usr/bin/g++"):
    NVCC_FLAGS += ["-ccbin", "/usr/bin/g++"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    deps.append(os.path.join(ROOT, "include", "thorx.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=True):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + sources()
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
