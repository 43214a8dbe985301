"""Build libradchan.so (sm_100a) in-tree with nvcc.

The library is plain C++/CUDA behind the C ABI of include/radchan.h; no
torch headers are involved.  Objects go to radchan_b200/_build/, the shared
library to radchan_b200/libradchan.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libradchan.so")
LIB_CHECKED = os.path.join(HERE, "libradchan_checked.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false and -ffp-contract=off keep device and host arithmetic
# identical to the CPU oracle (no fused multiply-add contraction).
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
          "-I" + INCLUDE, "-I" + CSRC]


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _deps_mtime():
    m = 0.0
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _compile(src, ptxas_verbose=False, build_dir=BUILD, defines=()):
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps_mtime()):
        return obj, ""
    flags = COMMON + ["-D" + d for d in defines]
    cmd = [NVCC] + ARCH + flags + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + flags + ["-x", "c++", "-c", src, "-o", obj]
    if ptxas_verbose and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(verbose: bool = False, ptxas_verbose: bool = False, checked: bool = False) -> str:
    """checked=True builds libradchan_checked.so: the same sources with
    RC_CHECKED=1, every table, field and partial-sum index of the march
    checked against its array (status bit 3 instead of a fault)."""
    build_dir = BUILD + ("_checked" if checked else "")
    lib = LIB_CHECKED if checked else LIB
    defines = ("RC_CHECKED=1",) if checked else ()
    os.makedirs(build_dir, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_verbose, build_dir, defines), srcs))
    objs = [o for o, _ in results]
    if verbose or ptxas_verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return lib


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv, checked="--checked" in sys.argv))
