"""Particle scattering (optional medium; the reference's Monte Carlo path has
none, its table generator tabulates the particles: nbcorrk/write_tables.cpp
writeP :204-260 and writeH :326-336, CDF law calc_prob.cpp:253-270).

CPU checks of the host tables and of the oracle's scattering path:
  * the natural logarithm behind the free path -ln(u), against libm;
  * the synthetic Henyey-Greenstein tables follow calc_prob.cpp's trapezoid
    law; particle files round trip and malformed ones are rejected;
  * a zero scattering coefficient changes nothing, bit for bit;
  * an isothermal enclosure still has Q = 0 with scattering;
  * a grey slab with isotropic and with forward (Henyey-Greenstein g = 0.6)
    scattering matches an independent discrete-ordinates solution
    (tests/dom_slab.py) within the Monte Carlo error, family-wise 3 sigma;
  * energy balance of a closed enclosure with scattering.
The device equals the oracle bit for bit (tests/test_gpu_scattering.py).
"""
import ctypes as C
import os

import numpy as np
import pytest
from scipy import stats

import dom_slab as D
import mc_stats as MS
from radchan_b200 import api
from radchan_b200 import workloads as W

SIGMA = 5.670373e-08


def _oracle():
    from oracle import oracle as O
    return O


def _probe(which, x):
    O = _oracle()
    f = O.lib().oracle_math_probe
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros_like(x)
    assert f(which, x.size, x.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double))) == 0
    return out


def test_logf_error_bound_over_every_uniform():
    # every value rc_u01 can produce: k * 2^-24, k = 1 .. 2^24
    u = (np.arange(1, (1 << 24) + 1, dtype=np.float64) * 2.0 ** -24).astype(np.float32).astype(np.float64)
    got = _probe(7, u)
    ref = np.log(u)
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    m = ref != 0
    assert np.max(np.abs(got[m] - ref[m]) / ulp[m]) <= 2.0
    assert got[-1] == 0.0  # log(1) exactly


def test_log_double_error_bound():
    x = np.exp(np.linspace(-700, 700, 200001))
    got = _probe(8, x)
    ref = np.log(x)
    assert np.max(np.abs(got - ref) / np.spacing(np.abs(ref))) <= 2.0


def _hg_trapezoid_cdf(g, th):
    # calc_prob.cpp:253-270: trapezoids of p(theta) sin(theta), normalised by the last
    p = (1 - g * g) / (1 + g * g - 2 * g * np.cos(th)) ** 1.5
    pr = 0.5 * np.diff(th) * (p[1:] + p[:-1]) * 0.5 * (np.sin(th[1:]) + np.sin(th[:-1])) * 0.5
    c = np.concatenate([[0.0], np.cumsum(pr)])
    return c / c[-1]


def test_synthetic_tables_follow_the_trapezoid_law():
    sc = api.Scattering.synthetic(nB=12, nQ=3, nA=91, ksca_lo=0.1, ksca_hi=10.0, g_lo=-0.3, g_hi=0.8, seed=5)
    a = sc.arrays()
    th = np.pi * np.arange(91) / 90
    assert np.allclose(a["theta"], th.astype(np.float32))
    assert sc.validate() == ""
    k = a["ksca"]
    assert np.all(k >= 0.1 * (1 - 1e-6)) and np.all(k <= 10.0 * (1 + 1e-6))
    assert np.all(k == k[:, :1])  # the same at every g point
    for b in range(12):
        cdf = a["phase_cdf"][b].astype(np.float64)
        # recover the band's g from the CDF: the one whose trapezoid law matches
        from scipy.optimize import minimize_scalar
        r = minimize_scalar(lambda g: np.max(np.abs(_hg_trapezoid_cdf(g, th) - cdf)), bounds=(-0.3, 0.8),
                            method="bounded", options={"xatol": 1e-10})
        assert r.fun < 2e-6, (b, r.x, r.fun)


def test_scattering_files_round_trip_and_reference_format(tmp_path):
    sc = api.Scattering.synthetic(nB=5, nQ=2, nA=37, ksca_lo=0.2, ksca_hi=3.0, g_lo=0.1, g_hi=0.7, seed=9)
    sc.write_dir(tmp_path)
    back = api.Scattering.read_dir(tmp_path, 5, 2)
    a, b = sc.arrays(), back.arrays()
    assert b["nA"] == 37
    for key in ("theta", "phase_cdf"):
        assert np.array_equal(a[key], b[key]), key
    assert np.allclose(a["ksca"], b["ksca"], rtol=1e-6)
    # files as the table generator writes them (writeP / writeH formats)
    d = tmp_path / "gen"
    d.mkdir()
    kabs = np.array([[0.5, 0.25], [1.5, 1.0]])
    ksca = np.array([[2.0, 4.0], [0.125, 0.5]])
    for j in range(2):
        with open(d / ("NarrBand%d.txt" % j), "w") as f:
            f.write("%le\t%le\t%le \n" % (1000.0 + j, 1010.0 + j, 1005.0 + j))
            f.write("".join(" %le\t" % v for v in kabs[j]) + "\n")
            f.write("".join(" %le\t" % v for v in ksca[j]))
    nA = 180
    th = np.arange(nA) * np.pi / nA  # the generator's angle grid (read_files.cpp:225)
    with open(d / "prob_scatt.txt", "w") as f:
        for i in range(2):
            c = _hg_trapezoid_cdf(0.3 * i, th)
            for t in range(nA):
                f.write("%le\t%le\t%le\n" % (th[t], 1005.0 + i, c[t]))
    r = api.Scattering.read_dir(d, 2, 2).arrays()
    assert r["nA"] == nA
    assert np.allclose(r["ksca"], ksca) and np.allclose(r["kabs"], kabs)
    assert np.allclose(r["theta"], th, rtol=1e-6)
    assert r["phase_cdf"][0, -1] == 1.0 and r["phase_cdf"][1, 0] == 0.0


def test_malformed_particle_files_are_rejected(tmp_path):
    sc = api.Scattering.synthetic(nB=3, nQ=2, nA=19)
    sc.write_dir(tmp_path)
    with pytest.raises(RuntimeError):
        api.Scattering.read_dir(tmp_path, 4, 2)  # NarrBand3.txt missing
    lines = open(tmp_path / "prob_scatt.txt").read().splitlines()
    open(tmp_path / "prob_scatt.txt", "w").write("\n".join(lines[:-1]) + "\n")  # one row short
    with pytest.raises(RuntimeError):
        api.Scattering.read_dir(tmp_path, 3, 2)


@pytest.mark.parametrize("what", ["nan_k", "neg_k", "theta_order", "theta_pi", "cdf_first", "cdf_last",
                                  "cdf_decreasing", "cdf_nan", "nA"])
def test_validate_rejects(what):
    nB, nQ, nA = 4, 2, 10
    k = np.full((nB, nQ), 1.0, np.float32)
    th = np.linspace(0, np.pi, nA).astype(np.float32)
    c = np.tile(np.linspace(0, 1, nA, dtype=np.float32), (nB, 1))
    assert api.Scattering.from_arrays(k, th, c).validate() == ""
    if what == "nan_k":
        k[1, 1] = np.nan
    elif what == "neg_k":
        k[2, 0] = -1.0
    elif what == "theta_order":
        th[3] = th[2]
    elif what == "theta_pi":
        th[-1] = 3.2
    elif what == "cdf_first":
        c[0, 0] = 0.01
    elif what == "cdf_last":
        c[3, -1] = 0.99
    elif what == "cdf_decreasing":
        c[2, 5] = c[2, 3]
        c[2, 4] = c[2, 6]
    elif what == "cdf_nan":
        c[1, 4] = np.nan
    elif what == "nA":
        th, c = th[:1], c[:, :1]
    msg = api.Scattering.from_arrays(k, th, c).validate()
    assert msg != ""


def _slab(photmax, kappa, nx=16, ny=4, toll=1e-6):
    p = W.channel_params(nx, ny, ny, grey=True, photmax=photmax, nVar=4, Tw=0.0, Te=0.0, fact_mesh=1.5)
    p.abscoeff = kappa
    p.Tw[0] = p.Tw[1] = 0.0
    p.toll = p.tollS = toll  # the cutoff's escape bias (< toll of the emission) far below the MC error
    T = np.full(api.field_shape(p), 1000.0, np.float32)
    T[:, :, 0] = -1000.0  # face averages 0: cold black walls
    T[:, :, -1] = -1000.0
    return p, T


def _grey_scattering(p, sigma_s, g, nA=181):
    th = np.linspace(0.0, np.pi, nA)
    cdf = D.hg_cdf(g, th)
    cdf = ((cdf - cdf[0]) / (cdf[-1] - cdf[0])).astype(np.float32)
    cdf[-1] = 1.0
    return dict(ksca=np.full((p.grey_nB, 1), sigma_s, np.float32), theta=th.astype(np.float32),
                phase_cdf=np.tile(cdf, (p.grey_nB, 1)))


def test_zero_scattering_coefficient_changes_nothing():
    O = _oracle()
    tabs = W.tables_nb(nB=20, nQ=4, nT=32)
    p = W.channel_params(12, 6, 4, photmax=32, nVar=2, nB=20, nQ=4, nT=32, levels=[(12, 6, 4), (6, 3, 2)],
                         maxs=[4, 100000], calcwalls=1, adiabw=1, adiabe=1)
    T = W.channel_field(p, seed=21)
    sc = dict(ksca=np.zeros((20, 4), np.float32), theta=np.linspace(0, np.pi, 9).astype(np.float32),
              phase_cdf=np.tile(np.linspace(0, 1, 9, dtype=np.float32), (20, 1)))
    a = O.solve(p, tabs, T, rpt=8)
    b = O.solve(p, tabs, T, rpt=8, scatter=sc)
    for key in ("q64", "var64", "qw64", "vw64"):
        assert np.array_equal(a[key], b[key]), key
    assert a["steps"] == b["steps"]


def test_isothermal_enclosure_with_scattering_has_zero_source():
    O = _oracle()
    tabs = W.tables_nb(nB=30, nQ=4, nT=32)
    p = W.channel_params(12, 6, 6, photmax=64, nVar=2, nB=30, nQ=4, nT=32, adiabw=1, adiabe=1, calcwalls=1)
    T = W.isothermal_field(p, 800.0)
    sc = api.Scattering.synthetic(nB=30, nQ=4, nA=61, ksca_lo=0.3, ksca_hi=5.0, g_lo=-0.5, g_hi=0.9, seed=3)
    o = O.solve(p, tabs, T, rpt=8, scatter=sc.arrays())
    scale = 4 * O.setup(p, tabs, T).kappamax * SIGMA * 800.0 ** 4
    assert np.nanmax(np.abs(o["q64"])) < 1e-5 * scale
    assert np.max(np.abs(o["qw64"])) < 1e-5 * SIGMA * 800.0 ** 4
    # scattering did happen: more steps than without it
    assert o["steps"] > O.solve(p, tabs, T, rpt=8)["steps"] * 1.2


@pytest.mark.parametrize("g", [0.0, 0.6])
def test_scattering_slab_matches_discrete_ordinates(g):
    O = _oracle()
    kappa, sigma_s = 0.5, 1.0
    p, T = _slab(8192, kappa)
    sc = _grey_scattering(p, sigma_s, g)
    o = O.solve(p, None, T, rpt=16, scatter=sc)
    x = api.grid_level(p, 0)["x"][1:-1].astype(np.float64)
    phase = None if g == 0.0 else D.henyey_greenstein(g)
    ref = D.solve(p.Lx, kappa, sigma_s, 1000.0, x, phase=phase)
    m, se = MS.plane_stats(o["q64"], np.sqrt(o["var64"]))
    zc = MS.aggregates(m, se, ref, np.zeros_like(ref))
    assert zc["ok"], (zc["z"], zc["threshold"])
    # the comparison has power: without scattering the source differs by
    # many standard errors
    ref0 = D.solve(p.Lx, kappa, 0.0, 1000.0, x)
    assert np.max(np.abs(ref0 - ref) / se) > 20.0


def test_discrete_ordinates_matches_exponential_integrals_without_scattering():
    from scipy.special import expn
    p, _ = _slab(64, 1.0)
    x = api.grid_level(p, 0)["x"][1:-1].astype(np.float64)  # the points the Monte Carlo tests compare at
    for kappa in (0.2, 1.0, 3.0):
        q = D.solve(p.Lx, kappa, 0.0, 1000.0, x)
        ref = 2 * kappa * SIGMA * 1e12 * (expn(2, kappa * x) + expn(2, kappa * (p.Lx - x)))
        assert np.max(np.abs(q - ref)) < 2e-5 * 4 * kappa * SIGMA * 1e12


def test_energy_balance_closed_enclosure_with_scattering():
    O = _oracle()
    tabs = W.tables_nb(nB=30, nQ=4, nT=32, logk_lo=-1.0, logk_hi=1.0)
    p = W.channel_params(16, 8, 8, grey=False, photmax=512, nVar=4, nB=30, nQ=4, nT=32, adiabw=1, adiabe=1,
                         calcwalls=1, Ly=2.0, Lz=2.0)
    T = W.channel_field(p, seed=3)
    sc = api.Scattering.synthetic(nB=30, nQ=4, nA=91, ksca_lo=0.5, ksca_hi=4.0, g_lo=0.0, g_hi=0.8, seed=8)
    o = O.solve(p, tabs, T, rpt=16, scatter=sc.arrays())
    g = api.grid_level(p, 0)
    dx = np.diff(g["xu"]).astype(np.float64)
    dy, dz = p.Ly / p.jmax, p.Lz / p.kmax
    vol = (dx[None, None, :] * dy * dz)
    area = dy * dz
    total = (o["q64"] * vol).sum() + o["qw64"].sum() * area
    var = (o["var64"] * vol ** 2).sum() + o["vw64"].sum() * area ** 2
    scale = (np.abs(o["q64"]) * vol).sum()
    assert abs(total) < 4.5 * np.sqrt(var) + 2e-3 * scale, (total, np.sqrt(var), scale)


def test_phase_guide_brackets_return_the_bisection_index():
    """The method of the device's angle search (restated here with numpy):
    guide[q] = first a >= 1 with cdf[a] > q/G (nA-1 if none), then a
    bisection over (guide[q] - 1, guide[q+1]] -- returns the index of a
    bisection over the whole table, for every uniform including the bucket
    edges q/G, the CDF values themselves and the largest float below 1, on
    CDFs with flat stretches, jumps and long tails."""
    from phase_tables import odd_phase_cdfs
    G = 64
    f32 = np.float32

    def bisect_all(c, u):
        lo, hi = 0, len(c) - 1
        while hi - lo > 1:
            mid = (lo + hi) >> 1
            if u < c[mid]:
                hi = mid
            else:
                lo = mid
        return hi

    def guided(c, guide, u):
        q = min(int(f32(u) * f32(G)), G - 1)
        lo, hi = int(guide[q]) - 1, int(guide[q + 1])
        while hi - lo > 1:
            mid = (lo + hi) >> 1
            if u < c[mid]:
                hi = mid
            else:
                lo = mid
        return hi

    for nA in (2, 3, 17, 91, 181):
        if nA == 2:
            cdfs = np.array([[0, 1]], np.float32)
        elif nA == 3:
            cdfs = np.array([[0, 0, 1], [0, 1, 1], [0, 0.5, 1]], np.float32)
        else:
            cdfs = odd_phase_cdfs(8, nA, nA)
        for c in cdfs:
            guide = []
            a = 1
            for q in range(G + 1):
                thr = f32(q) / f32(G)
                while a < nA - 1 and not (c[a] > thr):
                    a += 1
                guide.append(a)
            us = [f32(0), f32(np.nextafter(f32(1), f32(0)))]
            us += [f32(q) / f32(G) for q in range(G)]
            us += [f32(np.nextafter(f32(q) / f32(G), f32(0))) for q in range(1, G)]
            us += [x for x in c if x < 1] + [f32(np.nextafter(x, f32(0))) for x in c if 0 < x <= 1]
            us += list(np.random.default_rng(nA).random(2000).astype(np.float32))
            for u in us:
                assert guided(c, guide, u) == bisect_all(c, u), (nA, u)
