"""Run the reference's own CUDA solver (built by oracle/ref_build.py into
oracle/_ref/) on a B200 and store its per-cell results as statistical parity
fixtures:

  tests/golden/ref_grey32.npz  -- grey gas, 32^3 channel (kappa = 1/m, black
      walls 955 K / 573 K, periodic y/z, photmax 64, nVar 4): Q and sigma of
      every interior cell as returned by get_results_, the seed of the
      temperature field, and the wall-clock times of mc_gpu_+get_results_.

The reference resets the device inside get_results_, so every solve runs in a
child process of its own.  Usage (on a GPU machine):

    python tests/golden/make_ref_fixtures.py [--repeats 3]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELD_SEED = 7


def child(name, out_path):
    from radchan_b200 import api
    from radchan_b200 import workloads as W
    assert name == "grey32"
    p = W.config_grey_32()
    T = W.channel_field(p, seed=FIELD_SEED)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_%s.so" % name))
    lib.ref_solve.restype = C.c_int
    lib.ref_solve.argtypes = [C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                              C.POINTER(C.c_double)]
    Q = np.zeros(api.result_shape(p), np.float32)
    S = np.zeros(api.result_shape(p), np.float32)
    ms = C.c_double()
    Tc = np.ascontiguousarray(T)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    rc = lib.ref_solve(fp(Tc), 1, fp(Q), fp(S), C.byref(ms))
    np.savez(out_path, Q=Q[1:-1, 1:-1, 1:-1], sigma=S[1:-1, 1:-1, 1:-1], ms=ms.value, rc=rc)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--child", default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.child:
        child(a.child, a.out)
        return
    name = "grey32"
    runs = []
    for r in range(a.repeats):
        tmp = os.path.join(ROOT, "gpurun_out", "ref_%s_%d.npz" % (name, r))
        os.makedirs(os.path.dirname(tmp), exist_ok=True)
        subprocess.check_call([sys.executable, __file__, "--child", name, "--out", tmp])
        runs.append(np.load(tmp))
    first = runs[0]
    assert int(first["rc"]) == 0, "reference returned CUDA error %d" % int(first["rc"])
    # the reference seeds its generators identically on every call
    same = all(np.array_equal(first["Q"], r["Q"]) for r in runs[1:])
    meta = dict(config="grey32", field_seed=FIELD_SEED, ms=[float(r["ms"]) for r in runs], repeat_identical=same)
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), Q=first["Q"], sigma=first["sigma"],
                        meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
