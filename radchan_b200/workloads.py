"""Seeded synthetic workloads: the channel temperature field and the
parameter sets of the benchmark configurations.

The reference ships neither temperature fields nor spectral tables
(properties/*.txt are absent), so every input here is generated from a
seeded recipe:

  T(x,y,z) = [Tw + (Te - Tw) x/Lx] * (1 + 0.05 * sum_m a_m sin(2 pi (ky_m y/Ly
             + kz_m z/Lz) + phi_m)),   m = 1..8, (ky, kz) in {1..4}^2,
  sum |a_m| = 1, phases uniform on [0, 2 pi); x-ghost cells 2 T_wall - T_1
  (face average = wall temperature), y/z ghosts periodic images.

Correlated-k tables: k_{b,g}(T) = k0_b exp(1.5 xi_g) (T/1000)^{n_b} built by
rc_tables_synthetic.  The grid uses the reference's parabolic x stretching
dx = 0.5 - fact_mesh (r - 0.5)^2 (src/montecarlo/definitions.h:108-136).
"""
from __future__ import annotations

import numpy as np

from . import api


def channel_params(imax, jmax, kmax, *, grey=False, photmax=64, nVar=4, levels=None, maxs=None,
                   Lx=2.0, Ly=2 * np.pi, Lz=np.pi, fact_mesh=1.5, Tw=955.0, Te=573.0, adiabw=0, adiabe=0,
                   calcwalls=0, bd_y=1, bd_z=1, eps=1.0, nB=100, nQ=8, nT=64, srt=0, seed=1234,
                   chanHeight=1.0, floatpoint=0):
    p = api.default_params()
    p.imax, p.jmax, p.kmax = imax, jmax, kmax
    p.Lx, p.Ly, p.Lz = Lx, Ly, Lz
    p.fact_mesh = fact_mesh
    p.nVar, p.photmax = nVar, photmax
    p.chanHeight = chanHeight
    if levels is None:
        levels = [(imax, jmax, kmax)]
    if maxs is None:
        maxs = [5] * (len(levels) - 1) + [100000]
    api.set_levels(p, levels, maxs)
    p.num_gpu, p.p_col = 1, 1
    p.srt = srt
    p.grey = 1 if grey else 0
    p.calcwalls = calcwalls
    p.random = 0
    p.floatpoint = floatpoint
    for w in range(6):
        p.eps[w] = eps
        p.Tw[w] = 0.0
    p.Tw[0], p.Tw[1] = Tw, Te
    p.adiabw, p.adiabe = adiabw, adiabe
    p.bd[0], p.bd[1] = 2, 2
    p.bd[2], p.bd[3] = bd_y, bd_y
    p.bd[4], p.bd[5] = bd_z, bd_z
    p.toll = 1.0e-3
    p.tollS = 1.0e-3
    p.nB, p.nQ, p.nT = nB, nQ, nT
    p.seed = seed
    return p


def channel_field(p, seed=7, Tw=955.0, Te=573.0, amp=0.05, nmodes=8):
    """Temperature field (kmax+2, jmax+2, imax+2) float32, i fastest."""
    rng = np.random.default_rng(seed)
    g = api.grid_level(p, 0)
    x = g["x"].astype(np.float64)
    y = g["y"].astype(np.float64)
    z = g["z"].astype(np.float64)
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
    # x ghosts: face average equals the wall temperature
    T[:, :, 0] = 2 * Tw - T[:, :, 1]
    T[:, :, -1] = 2 * Te - T[:, :, -2]
    # y, z ghosts: periodic images
    T[:, 0, :] = T[:, -2, :]
    T[:, -1, :] = T[:, 1, :]
    T[0, :, :] = T[-2, :, :]
    T[-1, :, :] = T[1, :, :]
    return np.ascontiguousarray(T, dtype=np.float32)


def isothermal_field(p, T0):
    return np.full(api.field_shape(p), T0, np.float32)


# -------------------------------------------------------------- configs
def config_grey_32(photmax=64, nVar=4, **kw):
    """Grey gas, 32^3, kappa = 1/m, black walls at 955 K / 573 K, periodic y/z."""
    return channel_params(32, 32, 32, grey=True, photmax=photmax, nVar=nVar, **kw)


def config_nb_64(photmax=256, nVar=4, **kw):
    """Narrow-band 100x8, 64^3, 3 levels (64/32/16, maxs 5/5/1e5), srt=1,
    calcwalls=1 with an adiabatic west wall."""
    return channel_params(64, 64, 64, grey=False, photmax=photmax, nVar=nVar,
                          levels=[(64, 64, 64), (32, 32, 32), (16, 16, 16)], maxs=[5, 5, 100000],
                          srt=1, calcwalls=1, adiabw=1, adiabe=0, **kw)


def tables_nb(nB=100, nQ=8, nT=64, logk_lo=-3.0, logk_hi=2.0, seed=20240601):
    return api.TableSet.synthetic(nB=nB, nQ=nQ, nT=nT, T_lo=300.0, T_hi=2000.0, nu_lo=500.0, nu_hi=10000.0,
                                  logk_lo=logk_lo, logk_hi=logk_hi, nexp=1.0, kexp=1.5, seed=seed)


def config_precision(photmax=1024, nVar=8, floatpoint=0, **kw):
    """192x128x128, optically thick tables, eps 0.8, specular y walls,
    adiabatic x walls with wall fluxes."""
    return channel_params(192, 128, 128, grey=False, photmax=photmax, nVar=nVar, bd_y=3, eps=0.8,
                          adiabw=1, adiabe=1, calcwalls=1, floatpoint=floatpoint, **kw)


def batch_problems(n=64, seed=99, edges=(16, 24, 32, 48, 64, 96), photmaxes=(32, 128, 512)):
    """Uneven problems: edges per axis, half grey and half narrow-band
    (20-100 bands x 8 g), photmax per problem."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        im, jm, km = (int(rng.choice(edges)) for _ in range(3))
        grey = i % 2 == 0
        ph = int(rng.choice(photmaxes))
        nB = int(rng.integers(20, 101))
        p = channel_params(im, jm, km, grey=grey, photmax=ph, nVar=4, nB=nB, nQ=8, nT=64, seed=1000 + i)
        out.append(dict(params=p, grey=grey, nB=nB, field_seed=int(rng.integers(1, 1 << 30)),
                        table_seed=int(rng.integers(1, 1 << 30))))
    return out
