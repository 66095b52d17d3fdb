"""Builds gato_b200/libgato_b200.so (the CUDA library behind the C ABI) for
sm_100a with nvcc.  Usage: python -m gato_b200.build  (or import and call
build())."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgato_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "capi.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in
                  ("common.cuh", "dynamics.cuh", "stages.cuh", "kernels.cuh", "plant_tables.h")] + [
    os.path.join(ROOT, "include", "gato_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force=False, verbose=False, extra=None):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + (extra or []) + SOURCES + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(force=True, verbose=True, extra=extra))
