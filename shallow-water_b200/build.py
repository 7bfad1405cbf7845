"""Build libswcuda.so (sm_100a) in-tree with nvcc.

    python shallow-water_b200/build.py [--force] [--bounds-check] [--all]

--bounds-check builds the debug variant libswcuda_bc.so instead (-DSW_BOUNDS_CHECK:
every access through the library's shared access helpers is checked against the
registered device allocations, see csrc/sw_bc.cuh); --all builds both, side by side.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libswcuda.so")
LIB_BC = os.path.join(HERE, "libswcuda_bc.so")
SOURCES = ["sw_capi.cu", "sw_noalloc.cu", "sw_tridiag.cu"]
DEPS = ["sw_capi.cu", "sw_noalloc.cu", "sw_tridiag.cu", "sw_solver.cuh", "sw_fft2d.cuh", "sw_fft.cuh", "sw_core.cuh",
        "sw_bc.cuh", "sw_spectral_host.h"]
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


def needs_build(lib=LIB):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(HERE, "..", "include", "sw_cuda.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _cmd(bounds_check):
    out = LIB_BC if bounds_check else LIB
    extra = ["-DSW_BOUNDS_CHECK"] if bounds_check else []
    return [_nvcc()] + NVCC_FLAGS + extra + ["-o", out] + [os.path.join(CSRC, s) for s in SOURCES]


def build(force=False, verbose=True, bounds_check=False, both=False):
    """Build the library (or its bounds-check variant); with both, build each one
    that is out of date, the two nvcc runs side by side."""
    variants = [False, True] if both else [bounds_check]
    todo = [v for v in variants if force or needs_build(LIB_BC if v else LIB)]
    procs = []
    for v in todo:
        cmd = _cmd(v)
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
    codes = [p.wait() for p in procs]
    for v, c in zip(todo, codes):
        if c != 0:
            raise subprocess.CalledProcessError(c, _cmd(v))
    return LIB_BC if (bounds_check and not both) else LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, bounds_check="--bounds-check" in sys.argv, both="--all" in sys.argv)
