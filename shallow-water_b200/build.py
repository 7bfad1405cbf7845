"""Build libswcuda.so (sm_100a) in-tree with nvcc.

    python shallow-water_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libswcuda.so")
SOURCES = ["sw_capi.cu", "sw_noalloc.cu", "sw_tridiag.cu"]
DEPS = ["sw_capi.cu", "sw_noalloc.cu", "sw_tridiag.cu", "sw_solver.cuh", "sw_fft2d.cuh", "sw_fft.cuh", "sw_core.cuh", "sw_spectral_host.h"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "--extended-lambda",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    # device-side optimisation of the compilation unit runs on all host cores
    "-split-compile=0",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(HERE, "..", "include", "sw_cuda.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=True):
    if not force and not needs_build():
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
