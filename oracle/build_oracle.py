"""Build recipe for the FP64 CPU oracle (test infrastructure only).

Compiles oracle/mpm_oracle.cpp (3D step) and oracle/solid_mpm2d_oracle.cpp (2D solid) into
oracle/lib/libmpm_oracle.so with g++ -O3 and OpenMP for a portable x86-64-v2 target (the tests), and,
on request, oracle/lib/libmpm_oracle_native.so with -march=native on the machine that runs it (the
CPU-baseline timing).
The reference itself is JavaScript (no compiled sources), so there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, f) for f in ("mpm_oracle.cpp", "solid_mpm2d_oracle.cpp")]
OUT_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(OUT_DIR, "libmpm_oracle.so")


# The portable build (checked by the tests on any x86-64-v2 host, built here and carried to other
# machines) and the native build for CPU-baseline timing, compiled on the machine that times it.
PORTABLE_ISA = "-march=x86-64-v2"
NATIVE_ISA = "-march=native"


def _host_tag() -> str:
    """Short fingerprint of this host's CPU (model and feature flags): a native build made on one
    machine is never loaded on another whose CPU may lack its instructions."""
    import hashlib
    info = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.strip() == "" and info:
                    break
    except OSError:
        import platform
        info = platform.processor() + platform.machine()
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def native_path() -> str:
    return os.path.join(OUT_DIR, f"libmpm_oracle_native_{_host_tag()}.so")


def build(force: bool = False, native: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    out = native_path() if native else OUT
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in SRCS):
        return out
    tmp = out + f".{os.getpid()}.tmp"
    cmd = ["g++", "-O3", NATIVE_ISA if native else PORTABLE_ISA, "-std=c++17", "-fopenmp", "-fPIC", "-shared",
           "-fno-fast-math", "-o", tmp, *SRCS]
    subprocess.check_call(cmd)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, native="--native" in sys.argv))
