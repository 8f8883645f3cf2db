"""Build libfdk_b200.so in-tree for sm_100a with nvcc (no torch, no JIT cache).

Usage:  python -m fdk_b200.build        (or fdk_b200.build.build() from Python)

The library links the CUDA runtime statically, so it loads (and its host-only entry points
run) on a machine without a GPU or driver; CUDA calls then return FDK_ERR_NO_DEVICE.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfdk_b200.so")
SOURCES = ["geometry.cpp", "filter.cu", "filter_noalloc.cu", "bp.cu", "rtk.cu", "phantom.cu", "recon.cu",
           "probe.cu", "fproj.cu", "learn.cu", "io.cpp", "toeplitz.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "fdk.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", CSRC,
              "-I", os.path.join(HERE, "..", "include")]
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc(), *ARCH, *common, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", tmp, "-cudart", "static",
           "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
