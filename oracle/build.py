"""Build the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

g++ with -ffp-contract=off and no fast-math, so that its arithmetic matches
the device kernels (built with nvcc -fmad=false) operation for operation.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")
DEPS = [SRC, os.path.join(HERE, "oracle.h"), os.path.join(ROOT, "include", "radchan_math.h"),
        os.path.join(ROOT, "include", "radchan.h")]


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in DEPS):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), "-I" + HERE, SRC, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
