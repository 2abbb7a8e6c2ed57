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
# (source, extra nvcc flags): the FP64 kernels and the host code that
# computes their constants must not contract multiply-adds; the shifted
# low-precision kernels may.
UNITS = [("mplbgpu.cu", ["-fmad=false"]), ("kernels_f64.cu", ["-fmad=false"]),
         ("kernels_lp.cu", ["-fmad=true"]), ("noalloc.cu", ["-fmad=false"]),
         ("batch.cu", ["-fmad=false"]),
         ("nn/conv.cu", ["-fmad=true"]), ("nn/warmstart.cu", ["-fmad=true"]),
         ("plan.cpp", [])]
SOURCES = [os.path.join(CSRC, u) for u, _ in UNITS]
HEADERS = [os.path.join(CSRC, h) for h in ("kernels.cuh", "lattice.h",
                                            "plan.h", "launch.h",
                                            "launch_impl.cuh", "swap.cuh",
                                            "batch_kernels.cuh", "tma.cuh",
                                            "nn/umma.cuh", "nn/conv.cuh",
                                            "nn/conv_host.h")] + [
    os.path.join(HERE, "..", "include", h) for h in ("mplbgpu.h", "mplbnn.h")]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


BUILD_DIR = os.path.join(HERE, "_build")


def compile_commands():
    """One nvcc command per translation unit (objects in _build/)."""
    cmds = []
    for unit, flags in UNITS:
        obj = os.path.join(BUILD_DIR, unit.replace("/", "_") + ".o")
        cmds.append((obj, ["nvcc", "-O3", "-std=c++17", ARCH, "-lineinfo"] +
                     flags + ["-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                              "-c", os.path.join(CSRC, unit), "-o", obj]))
    return cmds


def nvcc_command(out=OUT):
    """All flags used for the library (for inspection and tests)."""
    cmd = []
    for _, c in compile_commands():
        cmd += c
    return cmd


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    cmds = compile_commands()
    procs = []
    for obj, cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    link = ["nvcc", "-shared", ARCH, "-o", OUT] + [o for o, _ in cmds]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
