"""Build of the native library ``libibisco_b200.so`` (sm_100a) in-tree.

nvcc cross-compiles for sm_100a without a GPU.  The kernels are compiled with
``--fmad=false`` (no contraction of a*b+c into FMA), IEEE division and square
root, so REAL*4 arithmetic rounds exactly as the reference's gfortran build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libibisco_b200.so")

SOURCES = ["ibg_device.cu", "host_setup.cpp", "ibg_static.cu", "ibg_server.cpp"]
HEADERS = ["ibg_common.cuh", "ibg_kernels.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-shared"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ibisco_gpu.h")]
    return srcs, [d for d in deps if os.path.exists(d)]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    _, deps = _inputs()
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if a source is newer than it; returns its path."""
    if not force and not needs_build():
        return LIB
    srcs, _ = _inputs()
    cmd = [_nvcc(), *ARCH, *FLAGS, "-I", INCLUDE, "-o", LIB, *srcs]
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, env=env)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
