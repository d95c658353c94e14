"""Builds the sm_100a CUDA library in-tree: quietmap_b200/libqm_b200.so.

nvcc cross-compiles for sm_100a without a GPU. The library exports the C ABI of
include/qm_batch.h; the Python binding (quietmap_b200.native) loads it with ctypes.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqm_b200.so")
SOURCES = ["qm_lib.cu", "qm_zwicker.cu", "qm_mlp.cu", "qm_formats.cpp", "qm_line.cu", "qm_distribution.cu"]
OBJ_DIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-rdc=false"]


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(cuda, "bin", "nvcc")
    return path if os.path.exists(path) else "nvcc"


def newest_input():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(os.path.dirname(HERE), "include")
    paths += [os.path.join(inc, f) for f in os.listdir(inc)]
    paths.append(__file__)
    return max(os.path.getmtime(p) for p in paths)


def newest_header():
    """The newest shared input: headers under csrc/ and include/, and this script."""
    inc = os.path.join(os.path.dirname(HERE), "include")
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths += [os.path.join(inc, f) for f in os.listdir(inc)]
    paths.append(__file__)
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    """Compiles each source whose object is older than it or than any header, then links."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_input():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = newest_header()
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        stale = (force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path), headers))
        if stale:
            cmd = [nvcc(), *ARCH, *FLAGS, "-c", path, "-o", obj + ".tmp"]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            os.replace(obj + ".tmp", obj)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)
