"""Known answers and invariants of the OERM Monte Carlo path, on the CPU
oracle (the device agrees with the oracle bit for bit, tests/test_gpu_parity.py).

  * isothermal enclosure: every OERM term is I_b(T)/I_b(T) - 1 = 0;
  * grey isothermal slab between cold black walls: div q = 2 kappa sigma T^4
    [E2(tau) + E2(tau_L - tau)] (Modest, Radiative Heat Transfer, plane-
    parallel medium), evaluated at the cell centres because every bundle of
    a cell starts at its centre (mc_gpu_noint.cu:117-122);
  * energy balance: sum Q V + sum q_w A = 0 in a closed enclosure;
  * symmetry of Q about the channel centre for a symmetric field;
  * specular y walls equal periodic y walls for a y-independent field.
"""
import numpy as np
import pytest
from scipy.special import expn

from radchan_b200 import api
from radchan_b200 import workloads as W

SIGMA = 5.670373e-08


def _oracle():
    from oracle import oracle as O
    return O


def test_isothermal_enclosure_has_zero_source():
    O = _oracle()
    tabs = W.tables_nb(nB=30, nQ=4, nT=32)
    for grey, t in ((True, None), (False, tabs)):
        p = W.channel_params(12, 6, 6, grey=grey, photmax=64, nVar=2, nB=30, nQ=4, nT=32, adiabw=1, adiabe=1,
                             calcwalls=1)
        T = W.isothermal_field(p, 800.0)
        o = O.solve(p, t, T, rpt=8)
        scale = 4 * O.setup(p, t, T).kappamax * SIGMA * 800.0 ** 4  # emission per unit volume
        # each term is (1/I_b) I_b - 1, i.e. 0 or -2^-24 in float
        assert np.nanmax(np.abs(o["q64"])) < 1e-5 * scale
        assert np.max(np.abs(o["qw64"])) < 1e-5 * SIGMA * 800.0 ** 4


def _slab_params(photmax, kappa=1.0, nx=16):
    p = W.channel_params(nx, 2, 2, grey=True, photmax=photmax, nVar=4, Tw=0.0, Te=0.0, fact_mesh=1.5)
    p.abscoeff = kappa
    p.Tw[0] = p.Tw[1] = 0.0
    return p


def _slab_field(p, T0=1000.0):
    T = np.full(api.field_shape(p), T0, np.float32)
    T[:, :, 0] = -T0   # face average 0: cold walls do not raise Tmax
    T[:, :, -1] = -T0
    return T


def slab_analytic(p, T0=1000.0):
    g = api.grid_level(p, 0)
    kap = p.abscoeff
    x = g["x"][1:-1].astype(np.float64)
    return 2 * kap * SIGMA * T0 ** 4 * (expn(2, kap * x) + expn(2, kap * (p.Lx - x)))


@pytest.mark.parametrize("kappa", [1.0, 0.2, 3.0, 1e-4])
def test_grey_slab_matches_exponential_integral_solution(kappa):
    O = _oracle()
    p = _slab_params(4096, kappa)
    T = _slab_field(p)
    o = O.solve(p, None, T, rpt=16)
    q = o["q64"].mean(axis=(0, 1))
    s = np.sqrt(o["var64"].mean(axis=(0, 1)) / 4)  # mean over the 4 cells of each plane
    ref = slab_analytic(p)
    emis = 4 * kappa * SIGMA * 1000.0 ** 4
    # rays are cut at transmissivity 1e-3 (the reference's toll), which biases
    # the escape fraction by at most ~1e-3 of the emission
    tol = 4.5 * s + 2e-3 * emis
    assert np.all(np.abs(q - ref) < tol), (q, ref, tol)


def test_energy_balance_closed_enclosure():
    O = _oracle()
    tabs = W.tables_nb(nB=30, nQ=4, nT=32, logk_lo=-1.0, logk_hi=1.0)
    p = W.channel_params(16, 8, 8, grey=False, photmax=512, nVar=4, nB=30, nQ=4, nT=32, adiabw=1, adiabe=1,
                         calcwalls=1, Ly=2.0, Lz=2.0)
    T = W.channel_field(p, seed=3)
    o = O.solve(p, tabs, T, rpt=16)
    g = api.grid_level(p, 0)
    dx = np.diff(g["xu"]).astype(np.float64)
    dy, dz = p.Ly / p.jmax, p.Lz / p.kmax
    vol = (dx[None, None, :] * dy * dz)
    area = dy * dz
    total = (o["q64"] * vol).sum() + o["qw64"].sum() * area
    var = (o["var64"] * vol ** 2).sum() + o["vw64"].sum() * area ** 2
    scale = (np.abs(o["q64"]) * vol).sum()
    assert abs(total) < 4.5 * np.sqrt(var) + 2e-3 * scale, (total, np.sqrt(var), scale)


def test_symmetry_about_channel_centre():
    O = _oracle()
    p = W.channel_params(16, 4, 4, grey=True, photmax=2048, nVar=4, Tw=900.0, Te=900.0)
    g = api.grid_level(p, 0)
    x = g["x"].astype(np.float64)
    prof = 900.0 + 300.0 * np.sin(np.pi * np.clip(x, 0, p.Lx) / p.Lx)
    T = np.broadcast_to(prof[None, None, :], api.field_shape(p)).astype(np.float32).copy()
    T[:, :, 0] = 2 * 900.0 - T[:, :, 1]
    T[:, :, -1] = 2 * 900.0 - T[:, :, -2]
    o = O.solve(p, None, T, rpt=16)
    q = o["q64"].mean(axis=(0, 1))
    s = np.sqrt(o["var64"].mean(axis=(0, 1)) / 16)
    assert np.all(np.abs(q - q[::-1]) < 4.5 * np.sqrt(s ** 2 + s[::-1] ** 2) + 1e-9)


def test_specular_y_equals_periodic_y_for_y_independent_field():
    O = _oracle()
    tabs = W.tables_nb(nB=20, nQ=4, nT=32)
    base = dict(grey=False, photmax=1024, nVar=4, nB=20, nQ=4, nT=32)
    p1 = W.channel_params(12, 6, 4, bd_y=1, **base)
    p3 = W.channel_params(12, 6, 4, bd_y=3, **base)
    T = W.channel_field(p1, seed=4)
    T[:] = T[:, 3:4, :]  # independent of y
    a = O.solve(p1, tabs, T, rpt=16)
    b = O.solve(p3, tabs, T, rpt=16)
    qa, qb = a["q64"].mean(axis=(0, 1)), b["q64"].mean(axis=(0, 1))
    s = np.sqrt((a["var64"].mean(axis=(0, 1)) + b["var64"].mean(axis=(0, 1))) / 24)
    assert np.all(np.abs(qa - qb) < 4.5 * s + 1e-9)
