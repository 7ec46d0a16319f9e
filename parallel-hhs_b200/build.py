"""Build recipe for libhhs_b200.so (CUDA kernels + C ABI), sm_100a only.

Objects go to _build/ next to this file and the shared library is written in-tree,
so it travels with the source tree. Rebuilds only what changed.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhhs_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = _headers()
    objs = []
    for s in srcs:
        o = os.path.join(OUT, os.path.basename(s) + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs) or ptxas_info:
            cmd = [NVCC] + ARCH + COMMON + ["-c", s, "-o", o]
            if ptxas_info and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


def build_compat_test(verbose=False):
    """Compiles tests/cpp/test_compat.cpp (a reference-style caller of include/hhs.hpp)."""
    src = os.path.join(ROOT, "tests", "cpp", "test_compat.cpp")
    out_dir = os.path.join(ROOT, "tests", "cpp", "_build")
    exe = os.path.join(out_dir, "test_compat")
    if not os.path.exists(src):
        return None
    os.makedirs(out_dir, exist_ok=True)
    if _newer(exe, [src, LIB] + _headers() + [os.path.join(ROOT, "include", "hhs.hpp")]):
        cmd = [NVCC] + ARCH + ["-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), src,
                               "-o", exe, "-L" + HERE, "-lhhs_b200", "-Xlinker",
                               "-rpath=$ORIGIN/../../../parallel-hhs_b200"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return exe


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas-info" in sys.argv)
    build_compat_test(verbose=True)
