"""Builds libmpm_b200.so (sm_100a) in-tree with nvcc.

    python summer-particle-lab_b200/build_lib.py [--force] [--verbose]

The library is a plain C-ABI shared object (include/mpm_b200.h); the CUDA runtime is linked
statically and the driver's tensor-map encoder is resolved at run time, so no libcuda link is
needed and the library loads on machines without a GPU.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libmpm_b200.so")
SOURCES = ["mpm_kernels.cu", "mpm_api.cu", "mpm_noalloc.cu", "solid2d.cu", "surrogate.cu", "pairs.cu"]
HEADERS = ["mpm_internal.h", "mpm_math.h", "pairs.h", "surrogate_net.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mpm_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    if not force and not _stale():
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false",
               "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
        objs.append(obj)
    subprocess.check_call([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"])
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
