"""Build the CUDA library librigidfibers.so in-tree (sm_100a).

    python -m rigidfibers_b200.build [--verbose]

Compiles rigidfibers_b200/csrc/*.cu with nvcc for sm_100a only and links
them into rigidfibers_b200/librigidfibers.so (kept out of git, shipped with
the working tree).
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librigidfibers.so")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The image's CXX points at a gcc without libgomp / full runtime; nvcc uses
# the system g++ as host compiler.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
         "--expt-relaxed-constexpr", "-ftz=true", "-Xptxas", "-warn-spills"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(HERE, "..", "include", "rigidfibers.h")]
    objs = []
    for src in sources:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(objs, OUT):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", OUT] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(OUT)
