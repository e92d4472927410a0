"""Builds thor_b200/libthorx.so (the CUDA kernels and the C ABI) for sm_100a with nvcc.

    python -m thor_b200.build [--force]   # or build() from __graft_entry__.py

Each source compiles to its own object (in parallel); the library links them. A second library,
libthorx_reforder.so, links the same objects except the dynamical-core kernels, which are
compiled with the reference's own operation order in the FP64 hyperdiffusion and divergence
damping (THORX_FP64_DIFF_WEIGHTS=0, THORX_FP64_DIVM_WEIGHTS=0) instead of the operator weights;
it exists for the parity test that keeps the two orders within rounding of each other.

Then thor_b200/bin/esp, the C++ program that runs a simulation from a .thr file (thor_b200/esp/),
is compiled with the host compiler against libthorx.so's C ABI (found through its run path).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libthorx.so")
LIB_REFORDER = os.path.join(HERE, "libthorx_reforder.so")
ESP_DIR = os.path.join(HERE, "esp")
ESP_BIN = os.path.join(HERE, "bin", "esp")
ESP_SOURCES = ["esp.cpp", "h5file.cpp"]

SOURCES = ["thorx_capi.cu", "dyn_fp64.cu", "rt.cu", "globdiag.cu", "surrogate.cu", "icogrid.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                 "-I" + os.path.join(ROOT, "include")]
LDFLAGS = ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-lgomp"]
REFORDER_DEFS = ["-DTHORX_FP64_DIFF_WEIGHTS=0", "-DTHORX_FP64_DIVM_WEIGHTS=0"]
# the environment's default host compiler may lack the OpenMP runtime; the system g++ has it
HOST = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def deps():
    d = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
         if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    d.append(os.path.join(ROOT, "include", "thorx.h"))
    d.append(os.path.abspath(__file__))
    return d


def esp_deps():
    return [os.path.join(ESP_DIR, f) for f in os.listdir(ESP_DIR)
            if f.endswith((".cpp", ".h"))] + [os.path.join(ROOT, "include", "thorx.h"), LIB]


def needs_build():
    if not (os.path.exists(LIB) and os.path.exists(LIB_REFORDER)):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(LIB_REFORDER))
    return any(os.path.getmtime(d) > t for d in deps())


def esp_needs_build():
    if not os.path.exists(ESP_BIN):
        return True
    t = os.path.getmtime(ESP_BIN)
    return any(os.path.getmtime(d) > t for d in esp_deps())


def build_esp(verbose=True):
    """thor_b200/bin/esp over libthorx.so (run path $ORIGIN/..)."""
    os.makedirs(os.path.dirname(ESP_BIN), exist_ok=True)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else os.environ.get("CXX", "g++")
    _run([cxx, "-O2", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"), "-o", ESP_BIN]
         + [os.path.join(ESP_DIR, s) for s in ESP_SOURCES]
         + ["-L" + HERE, "-l:libthorx.so", "-Wl,-rpath,$ORIGIN/.."], verbose)
    return ESP_BIN


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, end="", flush=True)


def build(force=False, verbose=True):
    if not force and not needs_build():
        if esp_needs_build():
            build_esp(verbose)
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    jobs = []  # (source, object, extra flags)
    for s in SOURCES:
        jobs.append((s, os.path.join(OBJ, s + ".o"), []))
    jobs.append(("dyn_fp64.cu", os.path.join(OBJ, "dyn_fp64_reforder.o"), REFORDER_DEFS))
    cmds = [[nvcc] + CFLAGS + HOST + extra + ["-c", "-o", o, os.path.join(CSRC, s)]
            for s, o, extra in jobs]
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    objs = [o for _, o, _ in jobs[:len(SOURCES)]]
    ref_objs = [jobs[-1][1] if s == "dyn_fp64.cu" else o
                for (s, o, _) in jobs[:len(SOURCES)]]
    _run([nvcc] + LDFLAGS + HOST + ["-o", LIB] + objs, verbose)
    _run([nvcc] + LDFLAGS + HOST + ["-o", LIB_REFORDER] + ref_objs, verbose)
    build_esp(verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
