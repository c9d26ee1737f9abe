"""Builds libpale_b200.so in-tree for sm_100a.

    python -m differentiablepointrendering_b200.build

The library is compiled with -fmad=false (host: -ffp-contract=off) so that
its vector arithmetic rounds like the host restatement of the algorithm.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ("csrc/build.cu", "csrc/render.cu", "csrc/optim.cu", "csrc/density.cu", "csrc/api.cu")
ARCH = ("-gencode", "arch=compute_100a,code=sm_100a")


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build_library(verbose: bool = False) -> str:
    out = os.path.join(HERE, "libpale_b200.so")
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(HERE, "..", "include", "pale_b200.h"))
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-o", out + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv))
