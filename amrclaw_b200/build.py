"""Build the in-tree CUDA library of the patch-advance path (sm_100a).

The library is compiled without FMA contraction (``--fmad=false`` on the device,
``-ffp-contract=off`` on the host) so that every FP64 result is bit-identical
to the CPU restatement used by the parity tests.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libamrgpu.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["kernels2d.cu", "noalloc2d.cu", "amr2d.cu", "kernels3d.cu", "flags3d.cu", "amr3d.cu", "amr1d.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(os.path.dirname(HERE), "include", "amrclaw_b200.h")
    return os.path.exists(hdr) and os.path.getmtime(hdr) > t


FLAGS = ["-std=c++17", "-O3", *ARCH, "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off"]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object (in parallel), then link the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(BUILD, exist_ok=True)

    def one(src: str) -> str:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *FLAGS, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, cwd=CSRC)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(one, SOURCES))
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
