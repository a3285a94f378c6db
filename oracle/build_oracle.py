"""Build recipe for the FP64 CPU oracle (test infrastructure only).

Compiles oracle/mpm_oracle.cpp (3D step) and oracle/solid_mpm2d_oracle.cpp (2D solid) into
oracle/lib/libmpm_oracle.so with g++ and OpenMP.
The reference itself is JavaScript (no compiled sources), so there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, f) for f in ("mpm_oracle.cpp", "solid_mpm2d_oracle.cpp")]
OUT_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(OUT_DIR, "libmpm_oracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(s) for s in SRCS):
        return OUT
    cmd = ["g++", "-O3", "-march=x86-64-v2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
           "-fno-fast-math", "-o", OUT, *SRCS]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
