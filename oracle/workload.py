"""The benchmark's seeded inputs built by the oracle alone (parameter set,
synthetic correlated-k tables, channel temperature field), so that the CPU
reference arm of bench.py runs without loading the product library.

TEST INFRASTRUCTURE ONLY.  tests/test_cpu_oracle_workload.py checks that
every input equals, byte for byte, the one radchan_b200/workloads.py builds
through libradchan.so.

  parameters  src/param/param.h defaults (the production channel,
              param.h:8-100, NarrowBand.h:189-219) with the channel
              overrides of the configuration;
  tables      oracle_tables_synthetic (oracle.cpp);
  field       T(x,y,z) = [Tw + (Te - Tw) x/Lx] (1 + 0.05 sum_m a_m
              sin(2 pi (ky_m y/Ly + kz_m z/Lz) + phi_m)), 8 modes, x ghosts
              2 T_wall - T_1, periodic y/z ghosts, on the grid of
              oracle_grid_level (definitions.h:68-136).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import abi
from oracle import oracle as O


def _default_params() -> abi.RcParams:
    """param.h / NarrowBand.h defaults (the reference's production channel)."""
    p = abi.RcParams()
    p.num_gpu, p.p_col = 1, 1
    p.imax, p.jmax, p.kmax = 406, 576, 2304
    p.Lx, p.Ly, p.Lz = 2.0, 6.283185307179586, 37.69911184307751
    p.fact_mesh = 1.6
    p.nVar, p.photmax = 1, 6000
    p.chanHeight = 0.5
    p.grid_num = 9
    mi = [406, 406, 406, 406, 406, 406 // 29, 406 // 29, 406 // 29, 406 // 203]
    mj = [576, 576 // 3, 576 // 6, 576 // 12, 576 // 24, 576 // 48, 576 // 96, 576 // 96, 576 // 192]
    mk = [2304 >> l for l in range(9)]
    for l in range(9):
        p.maxi[l], p.maxj[l], p.maxk[l] = mi[l], mj[l], mk[l]
        p.maxs[l] = 100000 if l == 8 else 5
    p.num_streams, p.blockdim, p.nblocks = 2, 128, 4096
    p.srt, p.grey, p.calcwalls, p.random, p.floatpoint = 1, 0, 0, 1, 0
    for w in range(6):
        p.eps[w], p.Tw[w] = 1.0, 0.0
    p.adiabw, p.adiabe = 1, 1
    p.stefan = 5.670373e-08
    p.toll, p.tollS = 1.0e-3, 1.0e-3
    for w, b in enumerate((2, 2, 1, 1, 4, 4)):
        p.bd[w] = b
    p.nT, p.nQ, p.nB = 135, 16, 999
    p.grey_nT, p.grey_nB = 65, 1000
    p.abscoeff, p.Tmins, p.wvmax = 1.0, 490.0, 5000.0
    p.seed = 1234
    return p


def channel_params(imax, jmax, kmax, *, grey=False, photmax=64, nVar=4, levels=None, maxs=None, adiabw=0,
                   adiabe=0, calcwalls=0, srt=0, nB=100, nQ=8, nT=64, seed=1234) -> abi.RcParams:
    """The channel of the benchmark configurations: Lx 2 (parabolic x
    stretching, fact_mesh 1.5), Ly 2 pi, Lz pi, black x walls at 955 K /
    573 K, periodic y and z, chanHeight 1, tolerances 1e-3."""
    p = _default_params()
    p.imax, p.jmax, p.kmax = imax, jmax, kmax
    p.Lx, p.Ly, p.Lz = 2.0, 2 * np.pi, np.pi
    p.fact_mesh = 1.5
    p.nVar, p.photmax = nVar, photmax
    p.chanHeight = 1.0
    levels = levels or [(imax, jmax, kmax)]
    maxs = maxs or [5] * (len(levels) - 1) + [100000]
    p.grid_num = len(levels)
    for l, (a, b, c) in enumerate(levels):
        p.maxi[l], p.maxj[l], p.maxk[l], p.maxs[l] = a, b, c, maxs[l]
    p.srt, p.grey, p.calcwalls, p.random, p.floatpoint = srt, 1 if grey else 0, calcwalls, 0, 0
    for w in range(6):
        p.eps[w], p.Tw[w] = 1.0, 0.0
    p.Tw[0], p.Tw[1] = 955.0, 573.0
    p.adiabw, p.adiabe = adiabw, adiabe
    for w, b in enumerate((2, 2, 1, 1, 1, 1)):
        p.bd[w] = b
    p.toll, p.tollS = 1.0e-3, 1.0e-3
    p.nB, p.nQ, p.nT = nB, nQ, nT
    p.seed = seed
    return p


def params_nb64(photmax=256, nVar=4) -> abi.RcParams:
    """Narrow-band 100x8, 64^3, 3 levels (64/32/16, maxs 5/5/1e5), srt 1,
    calcwalls with an adiabatic west wall."""
    return channel_params(64, 64, 64, photmax=photmax, nVar=nVar, levels=[(64, 64, 64), (32, 32, 32), (16, 16, 16)],
                          maxs=[5, 5, 100000], srt=1, calcwalls=1, adiabw=1, adiabe=0)


class Tables:
    """Synthetic tables held in numpy arrays, with an rc_tables view."""

    def __init__(self, nB=100, nQ=8, nT=64, T_lo=300.0, T_hi=2000.0, nu_lo=500.0, nu_hi=10000.0, logk_lo=-3.0,
                 logk_hi=2.0, nexp=1.0, kexp=1.5, seed=20240601):
        spec = abi.RcSynthSpec(nB, nQ, nT, T_lo, T_hi, nu_lo, nu_hi, logk_lo, logk_hi, nexp, kexp, seed)
        self.a = {n: np.zeros(s, np.float32) for n, s in
                  (("Tnb", nT), ("kP", nT), ("wvl", nB), ("wvr", nB), ("wvc", nB), ("kavg", nB),
                   ("kq", (nB, nT, nQ)), ("prob", (nT, nB)), ("probg", (nT, nB, nQ)), ("wq", nQ))}
        fp = lambda k: self.a[k].ctypes.data_as(C.POINTER(C.c_float))
        f = O.lib().oracle_tables_synthetic
        f.restype = C.c_int
        f.argtypes = [C.POINTER(abi.RcSynthSpec)] + [C.POINTER(C.c_float)] * 10
        rc = f(C.byref(spec), fp("Tnb"), fp("kP"), fp("wvl"), fp("wvr"), fp("wvc"), fp("kavg"), fp("kq"), fp("prob"),
               fp("probg"), fp("wq"))
        if rc != 0:
            raise RuntimeError("oracle_tables_synthetic failed")
        self.view = abi.RcTables(nT, nB, nQ, fp("Tnb"), fp("kP"), fp("wvl"), fp("wvr"), fp("wvc"), fp("kavg"),
                                 fp("kq"), fp("prob"), fp("probg"), fp("wq"))

    def arrays(self):
        return self.a


def tables_nb(nB=100, nQ=8, nT=64, logk_lo=-3.0, logk_hi=2.0, seed=20240601) -> Tables:
    return Tables(nB=nB, nQ=nQ, nT=nT, logk_lo=logk_lo, logk_hi=logk_hi, seed=seed)


def channel_field(p, seed=7, Tw=955.0, Te=573.0, amp=0.05, nmodes=8) -> np.ndarray:
    """Temperature field (kmax+2, jmax+2, imax+2) float32, i fastest."""
    rng = np.random.default_rng(seed)
    g = O.grid_level(p, 0)
    x, y, z = (g[n].astype(np.float64) for n in ("x", "y", "z"))
    ky = rng.integers(1, 5, nmodes)
    kz = rng.integers(1, 5, nmodes)
    ph = rng.uniform(0, 2 * np.pi, nmodes)
    a = rng.uniform(-1, 1, nmodes)
    a /= np.abs(a).sum()
    Z, Y = np.meshgrid(z, y, indexing="ij")
    f = np.zeros_like(Y)
    for m in range(nmodes):
        f += a[m] * np.sin(2 * np.pi * (ky[m] * Y / p.Ly + kz[m] * Z / p.Lz) + ph[m])
    prof = Tw + (Te - Tw) * x / p.Lx
    T = prof[None, None, :] * (1.0 + amp * f[:, :, None])
    T[:, :, 0] = 2 * Tw - T[:, :, 1]
    T[:, :, -1] = 2 * Te - T[:, :, -2]
    T[:, 0, :] = T[:, -2, :]
    T[:, -1, :] = T[:, 1, :]
    T[0, :, :] = T[-2, :, :]
    T[-1, :, :] = T[1, :, :]
    return np.ascontiguousarray(T, dtype=np.float32)


def nb64(photmax=256):
    """(params, tables, field) of the narrow-band 64^3 benchmark solve."""
    p = params_nb64(photmax=photmax)
    return p, tables_nb(), channel_field(p)


def write_reference_dir(tables: Tables, path: str) -> None:
    """Write the tables as the reference's readT reads them
    (read_tables.cpp:21-96; the formats of nbcorrk/write_tables.cpp:23-107):
    planck-mean.txt, prob_new2.txt and NarrBand%d.txt.  k_avg, which readT
    keeps from the last temperature row, is written on every row."""
    import os
    a = tables.arrays()
    nT, nB, nQ = a["Tnb"].size, a["wvc"].size, a["wq"].size
    os.makedirs(path, exist_ok=True)
    with open(os.path.join(path, "planck-mean.txt"), "w") as f:
        for i in range(nT):
            f.write("%f %e %e %e\n" % (a["Tnb"][i], a["kP"][i], 0.0, 0.0))
    with open(os.path.join(path, "prob_new2.txt"), "w") as f:
        for i in range(nT):
            for j in range(nB):
                f.write("%f \t %-5d \t%30.20e \t" % (a["Tnb"][i], j, a["prob"][i, j]))
                f.write("".join("%30.20e\t" % a["probg"][i, j, g] for g in range(nQ)))
                f.write("\n")
    for j in range(nB):
        with open(os.path.join(path, "NarrBand%d.txt" % j), "w") as f:
            f.write("%e\t%e\t%e \n" % (a["wvl"][j], a["wvr"][j], a["wvc"][j]))
            for i in range(nT):
                f.write(" %f\t %e\t %e\t" % (a["Tnb"][i], a["prob"][i, j], a["kavg"][j]))
                f.write("".join(" %e\t" % a["kq"][j, i, g] for g in range(nQ)))
                f.write("\n")
