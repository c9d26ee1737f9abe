"""Compiles the CPU oracle (test infrastructure) into oracle/_build/.

    python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle() -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libpale_oracle.so")
    srcs = [os.path.join(HERE, "pale_oracle.c"), os.path.join(HERE, "pale_oracle.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    cmd = ["gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-o", out + ".tmp", srcs[0], "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build_oracle())
