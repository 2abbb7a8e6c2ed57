"""Builds libmplbgpu.so (CUDA, sm_100a) in-tree.

    python -m mplb_b200.build

FP64 parity arithmetic needs -fmad=false on the device and
-ffp-contract=off on the host (plan.cpp computes boundary constants in the
reference's operation order).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmplbgpu.so")
SOURCES = [os.path.join(CSRC, "mplbgpu.cu"), os.path.join(CSRC, "noalloc.cu"),
           os.path.join(CSRC, "plan.cpp")]
HEADERS = [os.path.join(CSRC, h) for h in ("kernels.cuh", "lattice.h",
                                            "plan.h")] + [
    os.path.join(HERE, "..", "include", "mplbgpu.h")]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc_command(out=OUT, extra=()):
    return ["nvcc", "-O3", "-std=c++17", ARCH, "-lineinfo", "-fmad=false",
            "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-shared",
            "-o", out] + list(extra) + SOURCES


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    cmd = nvcc_command()
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
