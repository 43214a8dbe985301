"""Run the reference's own CUDA solver (built by oracle/ref_build.py into
oracle/_ref/) on a B200 and store its results as statistical parity
fixtures:

  tests/golden/ref_grey32.npz  -- grey gas, 32^3 channel (kappa = 1/m, black
      walls 955 K / 573 K, periodic y/z, photmax 64, nVar 4): Q and sigma of
      every interior cell as returned by get_results_, the seed of the
      temperature field, and the wall-clock times of mc_gpu_+get_results_.
  tests/golden/ref_nb64.npz    -- narrow-band 64^3 channel (100 bands x 8 g,
      64 temperatures of the seeded synthetic tables, 3 levels 64/32/16,
      photmax 256, nVar 4, adiabatic west wall with its flux).  From the
      srt = 0 build (independent replicates): per-x-plane means of Q and their
      standard errors, Q and sigma of 4096 sampled cells, and the west-wall
      flux and its sigma at every wall cell.  From the srt = 1 build (as the
      configuration states; its replicates share one band histogram per
      thread, so its sigma is biased low): per-x-plane means of Q with the
      standard errors it reports, and its west-wall flux and sigma at every
      wall cell.  From the srt = 0 build whose find_bandS edge rule is
      corrected ("nb64s0fix", oracle/ref_build.py): the west-wall flux and
      sigma at every wall cell.  Wall-clock times of the builds.

The reference resets the device inside get_results_ and reads its tables
from ./properties, so every solve runs in a child process of its own, in a
scratch directory holding the table files.  Usage (on a GPU machine):

    python tests/golden/make_ref_fixtures.py [--config grey32|nb64] [--repeats 3] [--outdir DIR]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELD_SEED = 7
NB_SAMPLE = 4096
NB_SAMPLE_SEED = 31


def problem(name):
    from radchan_b200 import workloads as W
    if name == "grey32":
        p = W.config_grey_32()
        return p, None, W.channel_field(p, seed=FIELD_SEED)
    p = W.config_nb_64()
    return p, W.tables_nb(), W.channel_field(p, seed=FIELD_SEED)


def child(name, lib_name, out_path, workdir):
    from radchan_b200 import api
    p, tabs, T = problem(name)
    if tabs is not None:
        os.makedirs(os.path.join(workdir, "properties"), exist_ok=True)
        tabs.write_dir(os.path.join(workdir, "properties"))
    os.chdir(workdir)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_%s.so" % lib_name))
    lib.ref_solve.restype = C.c_int
    lib.ref_solve.argtypes = [C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                              C.POINTER(C.c_double)]
    Q = np.zeros(api.result_shape(p), np.float32)
    S = np.zeros(api.result_shape(p), np.float32)
    ms = C.c_double()
    Tc = np.ascontiguousarray(T)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    rc = lib.ref_solve(fp(Tc), 1, fp(Q), fp(S), C.byref(ms))
    np.savez(out_path, Q=Q, sigma=S, ms=ms.value, rc=rc)


def run_children(name, lib_name, repeats, tmp):
    runs = []
    for r in range(repeats):
        out = os.path.join(tmp, "%s_%d.npz" % (lib_name, r))
        wd = tempfile.mkdtemp(dir=tmp)
        subprocess.check_call([sys.executable, __file__, "--child", name, "--lib", lib_name, "--out", out,
                               "--workdir", wd])
        runs.append(np.load(out))
        assert int(runs[-1]["rc"]) == 0, "reference returned CUDA error %d" % int(runs[-1]["rc"])
    same = all(np.array_equal(runs[0]["Q"], r["Q"]) for r in runs[1:])
    return runs, same


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="grey32", choices=["grey32", "nb64"])
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--child", default=None)
    ap.add_argument("--lib", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--outdir", default=HERE, help="where the .npz fixture is written")
    a = ap.parse_args()
    if a.child:
        child(a.child, a.lib, a.out, a.workdir)
        return
    tmp = tempfile.mkdtemp(prefix="rc_reffix_")
    if a.config == "grey32":
        runs, same = run_children("grey32", "grey32", a.repeats, tmp)
        Q = runs[0]["Q"][1:-1, 1:-1, 1:-1]
        S = runs[0]["sigma"][1:-1, 1:-1, 1:-1]
        meta = dict(config="grey32", field_seed=FIELD_SEED, ms=[float(r["ms"]) for r in runs], repeat_identical=same)
        np.savez_compressed(os.path.join(a.outdir, "ref_grey32.npz"), Q=Q, sigma=S, meta=json.dumps(meta))
        print(json.dumps(meta))
        return
    runs, same = run_children("nb64", "nb64s0", a.repeats, tmp)
    runs1, same1 = run_children("nb64", "nb64", a.repeats, tmp)
    runsf, samef = run_children("nb64", "nb64s0fix", a.repeats, tmp)

    def split(run):
        Qf = run["Q"].astype(np.float64)
        Sf = run["sigma"].astype(np.float64)
        Q, S = Qf[1:-1, 1:-1, 1:-1], Sf[1:-1, 1:-1, 1:-1]
        n = Q.shape[0] * Q.shape[1]
        # west-wall flux at i = 0 (get_results_ scatter, mc_gpu_noint.cu:996-1001)
        return Q, S, Q.mean(axis=(0, 1)), np.sqrt((S ** 2).sum(axis=(0, 1))) / n, Qf[1:-1, 1:-1, 0], Sf[1:-1, 1:-1, 0]

    Q, S, plane_mean, plane_se, wq, ws = split(runs[0])
    _, _, plane_mean1, plane_se1, wq1, ws1 = split(runs1[0])
    Qx, _, _, _, wqf, wsf = split(runsf[0])
    for name, arr in (("srt0 Q", Q), ("srt0 wall", wq), ("srt1 plane", plane_mean1), ("srt1 wall", wq1),
                      ("fixed-edge wall", wqf)):
        assert np.all(np.isfinite(arr)), "reference returned non-finite %s" % name
    rng = np.random.default_rng(NB_SAMPLE_SEED)
    flat = rng.choice(Q.size, size=NB_SAMPLE, replace=False)
    idx = np.stack(np.unravel_index(flat, Q.shape), axis=1).astype(np.int16)
    meta = dict(config="nb64", field_seed=FIELD_SEED, srt=0, ms=[float(r["ms"]) for r in runs],
                ms_srt1=[float(r["ms"]) for r in runs1], repeat_identical=same, repeat_identical_srt1=same1,
                repeat_identical_fix=samef, fix_fluid_identical=bool(np.array_equal(Qx, Q)),
                sample_seed=NB_SAMPLE_SEED, walls="west (adiabatic), kernel_surface emission patched")
    np.savez_compressed(os.path.join(a.outdir, "ref_nb64.npz"), plane_mean=plane_mean, plane_se=plane_se,
                        wall_q=wq.astype(np.float32), wall_sigma=ws.astype(np.float32),
                        sample_idx=idx, sample_Q=Q.reshape(-1)[flat], sample_sigma=S.reshape(-1)[flat],
                        srt1_plane_mean=plane_mean1, srt1_plane_se=plane_se1,
                        srt1_wall_q=wq1.astype(np.float32), srt1_wall_sigma=ws1.astype(np.float32),
                        fix_wall_q=wqf.astype(np.float32), fix_wall_sigma=wsf.astype(np.float32),
                        meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
