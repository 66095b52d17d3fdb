"""Builds oracle/_ref/libgrid_ref_<plant>.so: the reference's own dynamics,
plant cost and integrator headers compiled for the host in FP64.

Test infrastructure only.  The reference headers are read from where they lie
(reference_root(): $GATO_REF, else the recipe's default location); the GRiD headers are passed through a
filter that drops their CUDA kernel-launch host wrappers (functions whose body
contains a `<<<...>>>` launch) and their `__global__` kernels, which g++ cannot
parse and the oracle does not need.  The filtered tree lives in a temporary
directory that is removed after the build; only the shared libraries land in
oracle/_ref/.

Usage: python oracle/build_ref.py [plant ...]   (default: iiwa14 indy7)
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# The only place the reference tree's location is written: this recipe reads
# the reference's sources where they lie.  $GATO_REF overrides it.
DEFAULT_REF = "/root/reference"


def reference_root():
    """The reference source tree ($GATO_REF, else DEFAULT_REF), or None when
    neither holds it (nothing of oracle/_ref can be built then)."""
    root = os.environ.get("GATO_REF") or DEFAULT_REF
    return root if os.path.isdir(os.path.join(root, "gato")) else None


REF = reference_root() or (os.environ.get("GATO_REF") or DEFAULT_REF)

HEADERS = [
    "settings.h",
    "constants.h",
    "utils/linalg.cuh",
    "dynamics/integrator.cuh",
]


def _strip_comments(text):
    """Returns text with comments blanked (same length, newlines kept)."""
    out = list(text)
    i, n = 0, len(text)
    while i < n:
        if text.startswith("//", i):
            j = text.find("\n", i)
            j = n if j < 0 else j
            for k in range(i, j):
                out[k] = " "
            i = j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            j = n if j < 0 else j + 2
            for k in range(i, j):
                if out[k] != "\n":
                    out[k] = " "
            i = j
        elif text[i] == '"':
            j = i + 1
            while j < n and text[j] != '"':
                j += 2 if text[j] == "\\" else 1
            i = j + 1
        else:
            i += 1
    return "".join(out)


def filter_grid(text):
    """Drops namespace-level items that are __global__ kernels, launch a kernel,
    or are host-only launch wrappers (everything host-only except the model
    constant set-up)."""
    code = _strip_comments(text)
    depth = 0
    ns_depth = None
    items = []  # (start, end) of namespace-level items
    item_start = None
    i = 0
    n = len(code)
    while i < n:
        ch = code[i]
        if ns_depth is None:
            m = re.match(r"namespace\s+grid\s*\{", code[i:])
            if m:
                i += m.end()
                depth += 1
                ns_depth = depth
                item_start = i
                continue
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
            if ns_depth is not None and depth == ns_depth:
                items.append((item_start, i + 1))
                item_start = i + 1
            elif ns_depth is not None and depth < ns_depth:
                ns_depth = None
        elif ch == ";" and ns_depth is not None and depth == ns_depth:
            item_start = i + 1
        i += 1
    keep = ("init_XImats", "init_robotModel", "free_robotModel", "init_topology_helpers")
    drop = []
    for s, e in items:
        body = code[s:e]
        sig = body.split("{", 1)[0]
        host_only = re.search(r"\b__host__\b", sig) and not re.search(r"\b__device__\b", sig)
        if "<<<" in body or re.search(r"\b__global__\b", sig) or (
            host_only and not any(k in sig for k in keep)
        ):
            drop.append((s, e))
    out = []
    last = 0
    for s, e in drop:
        out.append(text[last:s])
        out.append("\n")
        last = e
    out.append(text[last:])
    return "".join(out)


def build(plant, program="grid_ref_wrap.cpp"):
    """Compiles ref_shim/<program> against the filtered reference headers:
    the shared library libgrid_ref_<plant>.so for grid_ref_wrap.cpp, the
    executable flop_count_<plant> for flop_count.cpp."""
    tmp = tempfile.mkdtemp(prefix="gato_ref_")
    try:
        gato = os.path.join(tmp, "gato")
        for rel in HEADERS + [
            f"dynamics/{plant}/{plant}_plant.cuh",
            f"dynamics/{plant}/{plant}_fext.cuh",
            f"dynamics/{plant}/{plant}_grid.cuh",
        ]:
            src = os.path.join(REF, "gato", rel)
            dst = os.path.join(gato, rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(src) as f:
                text = f.read()
            if rel.endswith("_grid.cuh"):
                text = filter_grid(text)
            with open(dst, "w") as f:
                f.write(text)
        os.makedirs(OUT, exist_ok=True)
        shared = program == "grid_ref_wrap.cpp"
        lib = os.path.join(OUT, f"libgrid_ref_{plant}.so" if shared else
                           f"{os.path.splitext(program)[0]}_{plant}")
        flag = "PLANT_IIWA14" if plant == "iiwa14" else "PLANT_INDY7"
        cmd = [
            "g++", "-std=c++17", "-O2", "-fPIC", "-w"] + (["-shared"] if shared else []) + [
            f"-D{flag}=1", "-DKNOT_POINTS=32", "-DNDEBUG",
            "-I", os.path.join(HERE, "ref_shim", "stub"),
            "-I", gato,
            "-include", "cuda_runtime.h",
            os.path.join(HERE, "ref_shim", program),
            "-o", lib,
        ]
        subprocess.run(cmd, check=True)
        return lib
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main(argv):
    plants = argv or ["iiwa14", "indy7"]
    if not os.path.isdir(os.path.join(REF, "gato")):
        print(f"reference tree not found at {REF}; nothing built")
        return 0
    for p in plants:
        print(build(p))
        print(build(p, "flop_count.cpp"))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
