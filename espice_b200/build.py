"""Builds libespice_lanes.so in-tree with nvcc for sm_100a.

The library is the product: CUDA kernels (csrc/kernels) and the C++ host
runtime behind the C ABI (csrc/host, include/espice_lanes.h). Device code
builds with --fmad=false and host code with -ffp-contract=off, so the
refactor, solves and stamps round as the reference's strict-float Zig.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libespice_lanes.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = [
    "csrc/host/sparse.cpp",
    "csrc/host/schedule.cpp",
    "csrc/host/records.cpp",
    "csrc/host/api.cpp",
    "csrc/host/lu_jit.cpp",
    "csrc/host/points.cpp",
    "csrc/kernels/newton.cu",
    "csrc/kernels/block.cu",
    "csrc/kernels/derive.cu",
    "csrc/kernels/mlp.cu",
    "csrc/host/mlp_host.cu",
]


def sources():
    return [os.path.join(HERE, s) for s in SOURCES]


def headers():
    inc = os.path.join(ROOT, "include")
    out = [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    for d in ("csrc", "csrc/host", "csrc/kernels"):
        p = os.path.join(HERE, d)
        out += [os.path.join(p, f) for f in os.listdir(p) if f.endswith((".h", ".hpp", ".cuh"))]
    return out


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


def _flags(verbose):
    return [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
            "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
            "-Xptxas", "-v" if verbose else "-O3"]


def build(force=False, verbose=False):
    """Compiles each source to an object in _build/ (in parallel), then links
    the shared library."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = [os.path.join(obj_dir, os.path.basename(s) + ".o") for s in sources()]

    def compile_one(i):
        return subprocess.run(_flags(verbose) + ["-c", sources()[i], "-o", objs[i]],
                              capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(objs)) as ex:
        results = list(ex.map(compile_one, range(len(objs))))
    for r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed building libespice_lanes.so")
        if verbose:
            sys.stderr.write(r.stderr)
    r = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs
                       + ["-lcudart", "-ldl", "-Xlinker", "--no-undefined"], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libespice_lanes.so")
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)
