"""Build the CUDA library in-tree: skmimageregistration_b200/_lib/libskm_b200.so.

nvcc cross-compiles for sm_100a only (no other architectures, no JIT PTX), so the
same command works on a machine without a GPU.  The library is a plain shared
object with the C-ABI of include/skm_gpu.h; Python reaches it through ctypes.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libskm_b200.so")
SOURCES = ["csrc/skm_capi.cu", "csrc/skm_noalloc.cu", "csrc/skm_conv.cu"]

def deps():
    """Every source the library is compiled from: all of csrc/ and the C headers."""
    files = glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
    files += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return files + [os.path.abspath(__file__)]


NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc()] + NVCC_FLAGS + [os.path.join(HERE, s) for s in SOURCES] + ["-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd, cwd=HERE)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
