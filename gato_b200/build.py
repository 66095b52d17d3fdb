"""Builds gato_b200/libgato_b200.so (the CUDA library behind the C ABI) for
sm_100a with nvcc.  Usage: python -m gato_b200.build  (or import and call
build())."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgato_b200.so")
CSRC = os.path.join(HERE, "csrc")
SOURCES = [os.path.join(CSRC, f) for f in ("capi.cu", "mixed.cu")]
DEPS = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
        if f.endswith((".cu", ".cuh", ".h"))] + [os.path.join(ROOT, "include", "gato_b200.h")]

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
    """Compiles every translation unit in parallel, then links the library."""
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    flags = [f for f in NVCC_FLAGS if f != "-shared"] + (extra or [])
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.basename(src) + ".o")
        cmd = [nvcc] + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    failed = [p for p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(failed[0].returncode, "nvcc")
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared"] + objs + [
        "-o", LIB + ".tmp"]
    subprocess.run(link, check=True)
    for o in objs:
        os.remove(o)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(force=True, verbose=True, extra=extra))
