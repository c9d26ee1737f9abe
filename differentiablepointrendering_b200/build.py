"""Builds libpale_b200.so in-tree for sm_100a.

    python -m differentiablepointrendering_b200.build
    PALE_NVCC_FLAGS="-DPALE_REFILL_STEPS=32" python -m differentiablepointrendering_b200.build

The library is compiled with -fmad=false (host: -ffp-contract=off) so that
its vector arithmetic rounds like the host restatement of the algorithm.
PALE_NVCC_FLAGS adds nvcc flags, typically the kernels' tuning knobs
(-DPALE_TOP_NODES, -DPALE_SMEM_STACK, -DPALE_GATHER_HITS, the register
budgets -DPALE_*_MIN_BLOCKS, -DPALE_REFILL_STEPS); the flags of the last
build are kept beside the library, and a different set rebuilds it.
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


def _read(path: str) -> str:
    try:
        with open(path) as f:
            return f.read()
    except OSError:
        return ""


def build_library(verbose: bool = False) -> str:
    out = os.path.join(HERE, "libpale_b200.so")
    stamp = out + ".flags"
    extra = os.environ.get("PALE_NVCC_FLAGS", "").split()
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(HERE, "..", "include", "pale_b200.h"))
    same_flags = _read(stamp) == " ".join(extra)
    if same_flags and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", *extra, "-o", out + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    with open(stamp, "w") as f:
        f.write(" ".join(extra))
    return out


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv))
