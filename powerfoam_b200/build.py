"""Build libpfoam.so (the C-ABI CUDA library) in-tree for sm_100a.

    python -m powerfoam_b200.build [--force]

All kernels are compiled with -fmad=false (plus the default IEEE division and
square root): the render kernels reproduce the reference's float32
expression sequence exactly, see csrc/pf_common.cuh.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libpfoam.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["pf_api.cu", "pf_bin.cu", "pf_composite.cu", "pf_batch.cu", "pf_raster.cu", "pf_trace.cu", "pf_adjacency.cu", "pf_interpen.cu",
           "pf_color.cu", "pf_mlp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _ccbin():
    for c in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return ["-ccbin", c]
    return []


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "pfoam.h"))
    return files


def needs_build():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    nvcc = _nvcc()
    for src in SOURCES:
        obj = os.path.join(LIB_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *FLAGS, *_ccbin(), "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call([nvcc, *ARCH, *_ccbin(), "-shared", "-o", tmp, *objs, "-lcudart"])
    os.replace(tmp, LIB_PATH)
    for o in objs:
        os.remove(o)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
