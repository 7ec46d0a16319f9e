"""Build recipe for the checker side (TEST INFRASTRUCTURE ONLY).

* liboracle_hhs.so -- the CPU FP64 restatement (hhs_oracle.c), gcc, no FMA contraction.
* _ref/            -- the reference's own code compiled from its source tree, where that
                      tree is present: the CPU split of src/cpu_scan.h (g++) and the GPU
                      scan / timestep / kick / drift of src/hold.cuh (nvcc, sm_100a, with
                      -fmad=false so its FP64 arithmetic is plain IEEE operations).
                      Outputs go only to _ref/ (git-ignored; it travels with the tree).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle():
    sys.path.insert(0, HERE)
    import oracle  # noqa: E402
    return oracle.build()


def reference_root_default():
    """The reference tree: $HHS_REFERENCE_ROOT, else a checkout named `reference` beside
    this repository's root."""
    return os.environ.get("HHS_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def build_ref(reference_root=None, verbose=False):
    """Compiles the reference shims if the reference tree exists; returns built paths."""
    if reference_root is None:
        reference_root = reference_root_default()
    src = os.path.join(reference_root, "src")
    if not os.path.isdir(src):
        return []
    os.makedirs(REF_OUT, exist_ok=True)
    built = []
    cpu_shim = os.path.join(HERE, "ref", "ref_cpu_shim.cpp")
    cpu_lib = os.path.join(REF_OUT, "libref_cpu.so")
    if _newer(cpu_lib, [cpu_shim, os.path.join(src, "cpu_scan.h")]):
        cmd = ["g++", "-O2", "-fPIC", "-shared", "-I" + src, "-o", cpu_lib, cpu_shim]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    built.append(cpu_lib)
    gpu_shim = os.path.join(HERE, "ref", "ref_gpu_shim.cu")
    gpu_lib = os.path.join(REF_OUT, "libref_gpu_nofma.so")
    deps = [gpu_shim] + [os.path.join(src, f) for f in os.listdir(src)]
    if _newer(gpu_lib, deps):
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-fmad=false",
               "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "20054", "-I" + src,
               "-o", gpu_lib, gpu_shim]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    built.append(gpu_lib)
    return built


if __name__ == "__main__":
    print(build_oracle())
    print(build_ref(verbose=True))
