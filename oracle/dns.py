"""CPU restatement of the channel DNS's use of a finished solve.

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py's CPU legs, never
by the product package.

Follows, in numpy double precision (IEEE, no contraction):
  src/dns/fixvar.f:1-14     read_kP: Tnb and kP from planck-mean.txt, kP * Height
  src/dns/fixvar.f:179-242  fix_rad: Qnew = Q/stefan/Tin**4, walls also /Height,
                            Varnew = sigma/stefan/Tin**4, the rank's j pencil
  src/dns/fixvar.f:16-43    fix_kappa + linear_int: Knew = kP at T1*Tin,
                            t = int(x0 - x(1)) / int(x(2) - x(1)) + 1
  src/dns/channel.f:260-266 Qnew *= underrelax; Gnew = 4*T1**4 - Qnew/Knew
Inputs are the Fortran-layout float Q and sigma that get_results_ returns,
(kloc+2, jmax+2, imax+2) with i fastest; T1 is the DNS pencil
(kloc+2, jn+2, imax+2); outputs are (kloc, jn, imax+2).

Where linear_int's row falls outside the table the reference reads past its
arrays; this restatement (like the library) extends the end interval and
counts the cell.  T1**4 is (T1*T1)*(T1*T1).
"""
from __future__ import annotations

import numpy as np


def read_kp(path, n, height):
    """fixvar.f:1-14: the first n rows of planck-mean.txt (T kP kR kM)."""
    rows = np.loadtxt(path, dtype=np.float64)[:n]
    return rows[:, 0].copy(), rows[:, 1] * height


def dns_source(Q, sigma, T1, Tin, Height, underrelax, stefan, Tnb, kP, jstart, jend):
    Tnb = np.asarray(Tnb, np.float64)
    kP = np.asarray(kP, np.float64)
    nT = len(Tnb)
    Tin4 = float(Tin) ** 4.0
    q = np.asarray(Q, np.float32)[1:-1, jstart:jend + 1, :].astype(np.float64)
    s = np.asarray(sigma, np.float32)[1:-1, jstart:jend + 1, :].astype(np.float64)
    Qn = q / stefan / Tin4
    Qn[:, :, 0] = Qn[:, :, 0] / Height
    Qn[:, :, -1] = Qn[:, :, -1] / Height
    Vn = s / stefan / Tin4
    T = np.asarray(T1, np.float64)[1:-1, 1:-1, :]
    x0 = T * Tin
    d = x0 - Tnb[0]
    dT = int(Tnb[1] - Tnb[0])
    ok = (d > -2147483648.0) & (d < 2147483648.0)
    ti = np.trunc(np.where(ok, d, 0.0)).astype(np.int64)
    t = np.sign(ti) * (np.abs(ti) // dT)          # Fortran integer division truncates
    t = np.where(ok, t, np.where(d > 0, nT, -1))
    clamped = int(((t < 0) | (t > nT - 2)).sum())
    t = np.clip(t, 0, nT - 2)
    slope = (kP[1:] - kP[:-1]) / (Tnb[1:] - Tnb[:-1])
    K = slope[t] * (x0 - Tnb[t]) + kP[t]
    Qn = Qn * underrelax
    t2 = T * T
    G = 4.0 * (t2 * t2) - Qn / K
    return dict(Qnew=Qn, Varnew=Vn, Knew=K, Gnew=G, n_clamped=clamped)
