"""Builds the reference's own CUDA solver module, unmodified, for sm_100a:
oracle/_ref/bsqpN<N>_<plant><ext>.so, the pybind11 module that the
reference's python/bsqp/interface.py imports (python/bindings.cu compiled with
the flags of the reference's CMakeLists.txt release build: -O3
-use_fast_math, KNOT_POINTS and PLANT_* definitions).

This is a measurement baseline, not the oracle: it is FP32 with fast math.
nvcc is run directly on the reference's python/bindings.cu where it lies
(build_ref.reference_root()); nothing is copied.  One module takes
several minutes to compile.

Only the FP32 build is made: the reference's USE_DOUBLES build raised an
illegal-address fault on the B200 and is not built or run.

Usage: python oracle/build_ref_gpu.py [plant:N ...]   (default: iiwa14:32)
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, HERE)
from build_ref import reference_root  # noqa: E402

REF = reference_root()


def module_path(plant, N):
    return os.path.join(OUT, f"bsqpN{N}_{plant}{sysconfig.get_config_var('EXT_SUFFIX')}")


def build(plant, N, force=False):
    out = module_path(plant, N)
    if REF is None:
        raise FileNotFoundError("reference tree not found: set GATO_REF to its location")
    src = os.path.join(REF, "python", "bindings.cu")
    if not os.path.exists(src):
        raise FileNotFoundError(f"reference source {src} not present")
    if os.path.exists(out) and not force:
        return out
    import pybind11
    os.makedirs(os.path.dirname(out), exist_ok=True)
    define = {"iiwa14": "PLANT_IIWA14=1", "indy7": "PLANT_INDY7=1"}[plant]
    cmd = ["nvcc", "-std=c++17", "-O3", "-use_fast_math",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC",
           f"-D{define}", f"-DKNOT_POINTS={N}",
           "-I", os.path.join(REF, "gato"),
           "-I", pybind11.get_include(),
           "-I", sysconfig.get_paths()["include"],
           src, "-o", out + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def main(argv):
    specs = argv or ["iiwa14:32"]
    for spec in specs:
        plant, N = spec.split(":")
        print(build(plant, int(N)))


if __name__ == "__main__":
    main(sys.argv[1:])
