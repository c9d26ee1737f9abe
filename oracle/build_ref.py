"""Compiles the reference renderer's own kernel sources for the CPU into
oracle/_ref/libpale_ref.so (test infrastructure).

    python oracle/build_ref.py <path of the reference checkout>

The sources are compiled where they lie, unmodified:
Pale/Renderer/Kernels/{PrimalKernels,AdjointKernels,PostprocessKernel}.cpp
and the headers they include, against the project's host SYCL subset
(oracle/ref_shim/), with oracle/ref_driver.cpp (the host flow of
SyclBridge.cpp / PathTracer.cpp / pale_bindings.cpp restated around them)
and the C oracle (scene build).  The library is a build product: it is
listed in .gitignore and travels to a GPU host beside the other built
libraries; nothing is copied from the reference into the repository.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libpale_ref.so")
KERNELS = ("PrimalKernels.cpp", "AdjointKernels.cpp", "PostprocessKernel.cpp")
FLAGS = ("-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC")


def sources(ref: str):
    pale = os.path.join(ref, "Pale")
    return [os.path.join(pale, "Renderer", "Kernels", k) for k in KERNELS]


def build_ref(ref: str, verbose: bool = False) -> str:
    pale = os.path.join(ref, "Pale")
    ref_srcs = sources(ref)
    for p in ref_srcs:
        if not os.path.exists(p):
            raise FileNotFoundError(p)
    own = [os.path.join(HERE, "ref_driver.cpp"), os.path.join(HERE, "ref_shim", "sycl_shim.cpp")]
    deps = ref_srcs + own + [os.path.join(HERE, "pale_oracle.c"), os.path.join(HERE, "pale_oracle.h"),
                             os.path.join(HERE, "ref_shim", "sycl", "sycl.hpp")]
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    inc = ["-I", os.path.join(HERE, "ref_shim"), "-I", pale, "-I", HERE]
    for src in ref_srcs + own:
        obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
        cmd = ["g++", "-std=c++20", *FLAGS, *inc, "-w", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cobj = os.path.join(OUT_DIR, "pale_oracle.o")
    subprocess.run(["gcc", "-std=c11", "-D_GNU_SOURCE", *FLAGS, "-c", os.path.join(HERE, "pale_oracle.c"), "-o", cobj],
                   check=True)
    objs.append(cobj)
    subprocess.run(["g++", "-shared", "-fopenmp", "-o", OUT + ".tmp", *objs, "-lm"], check=True)
    os.replace(OUT + ".tmp", OUT)
    for o in objs:
        os.unlink(o)
    return OUT


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    print(build_ref(sys.argv[1], verbose=True))
