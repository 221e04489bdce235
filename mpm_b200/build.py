"""Build recipe for libmpm_b200.so (sm_100a) with nvcc.

The library is built in-tree (mpm_b200/_lib/) so that it travels with the
source tree; the CUDA runtime is linked statically so the library does not
depend on which libcudart another module of the process loaded first.

    python -m mpm_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libmpm_b200.so")
RUNNER = os.path.join(LIBDIR, "mpm_gpu_run")
CXX = os.environ.get("CXX", "g++")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]

# (source, extra flags): the FP64 kernels never fuse multiply-add so that they
# round like the reference's scalar arithmetic; the mixed-precision kernels do.
UNITS = [
    ("kernels_fp64.cu", ["--fmad=false"]),
    ("kernels_mixed.cu", []),
    ("mpm_gpu.cu", []),
    ("noalloc.cu", []),
    ("pod.cu", []),
    ("kernels_tangent.cu", ["--fmad=false"]),
    ("kernels_adjoint.cu", ["--fmad=false"]),
    ("h5table.cpp", []),
]
HEADERS = ["mpm_math.cuh", "mpm_state.cuh", "mpm_kernels.h", "json_lite.hpp", "mpm_device.cuh", "mpm_bulk.cuh", "mpm_dual.cuh", "mpm_return.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "mpm_gpu.h")]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    # the C++ host driver over the C ABI (reads the reference's input files)
    src = os.path.join(HERE, "host", "mpm_gpu_run.cpp")
    if force or _newer(RUNNER, [src, LIB] + hdrs):
        cmd = [CXX, "-O2", "-std=c++17", "-Wall", "-pthread", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
               src, "-o", RUNNER, "-L", LIBDIR, "-lmpm_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
