"""DNS coupling on the CPU: the numpy restatement of fix_rad / fix_kappa /
the Gnew loop equals a statement-by-statement loop translation of the
Fortran (src/dns/fixvar.f:16-43, :179-242; channel.f:260-266), including
linear_int's truncating row rule and rows outside the table; read_kP
reads the table files the library writes."""
import math
import os

import numpy as np
import pytest

from oracle import dns as OD
from radchan_b200 import api
from radchan_b200 import workloads as W


def _loops(Q, S, T1, Tin, Height, underrelax, stefan, Tnb, kP, jstart, jend):
    """The Fortran loops with 0-based numpy indices [k][j][i]; Python floats
    are IEEE doubles, so every statement rounds as the Fortran's does."""
    kl = Q.shape[0] - 2
    nx = Q.shape[2]
    jn = jend - jstart + 1
    out = {k: np.zeros((kl, jn, nx)) for k in ("Qnew", "Varnew", "Knew", "Gnew")}
    n = len(Tnb)
    clamped = 0
    tin4 = Tin ** 4.0
    for k in range(1, kl + 1):
        for j in range(jstart, jend + 1):
            jl = j - jstart
            for i in range(nx):
                q = float(Q[k, j, i])
                out["Qnew"][k - 1, jl, i] = q / stefan / tin4                       # fixvar.f:205
                if i == 0 or i == nx - 1:
                    out["Qnew"][k - 1, jl, i] = q / stefan / tin4 / Height          # fixvar.f:211-212
                out["Varnew"][k - 1, jl, i] = float(S[k, j, i]) / stefan / tin4     # fixvar.f:225
    for k in range(1, kl + 1):
        for jl in range(1, jn + 1):
            for i in range(nx):
                x0 = float(T1[k, jl, i]) * Tin                                     # fixvar.f:25
                d = x0 - Tnb[0]
                if d != d or abs(d) >= 2147483648.0:
                    t = n if d > 0 else 0
                else:
                    a, b = int(d), int(Tnb[1] - Tnb[0])                             # fixvar.f:40
                    t = int(abs(a) // b) * (1 if a >= 0 else -1) + 1
                if t < 1 or t > n - 1:
                    clamped += 1
                    t = min(max(t, 1), n - 1)
                t -= 1
                y0 = (kP[t + 1] - kP[t]) / (Tnb[t + 1] - Tnb[t]) * (x0 - Tnb[t]) + kP[t]   # fixvar.f:41
                out["Knew"][k - 1, jl - 1, i] = y0
                qn = out["Qnew"][k - 1, jl - 1, i] * underrelax                     # channel.f:263
                out["Qnew"][k - 1, jl - 1, i] = qn
                t1 = float(T1[k, jl, i])
                out["Gnew"][k - 1, jl - 1, i] = 4.0 * ((t1 * t1) * (t1 * t1)) - qn / y0   # channel.f:264
    out["n_clamped"] = clamped
    return out


def _case(seed, im=6, jm=5, kl=3, jstart=2, jend=4, nT=9, step=26.98, spread=0.25):
    rng = np.random.default_rng(seed)
    Q = (rng.standard_normal((kl + 2, jm + 2, im + 2)) * 1e5).astype(np.float32)
    S = np.abs(rng.standard_normal((kl + 2, jm + 2, im + 2)) * 1e3).astype(np.float32)
    Tin = 955.0
    jn = jend - jstart + 1
    # temperatures around the table, some beyond either end
    T1 = (0.75 + spread * rng.standard_normal((kl + 2, jn + 2, im + 2)))
    Tnb = 300.0 + step * np.arange(nT)
    kP = np.exp(rng.standard_normal(nT)) * 0.5
    return dict(Q=Q, S=S, T1=T1, Tin=Tin, Height=0.5, underrelax=0.7, stefan=5.67e-08, Tnb=Tnb, kP=kP,
                jstart=jstart, jend=jend)


@pytest.mark.parametrize("seed,kw", [(1, {}), (2, dict(step=1.5, nT=40)), (3, dict(jstart=1, jend=5)),
                                     (4, dict(spread=2.0)), (5, dict(nT=2, step=400.0))])
def test_restatement_equals_fortran_loops_bit_for_bit(seed, kw):
    c = _case(seed, **kw)
    a = OD.dns_source(c["Q"], c["S"], c["T1"], c["Tin"], c["Height"], c["underrelax"], c["stefan"], c["Tnb"],
                      c["kP"], c["jstart"], c["jend"])
    b = _loops(c["Q"], c["S"], c["T1"], c["Tin"], c["Height"], c["underrelax"], c["stefan"], c["Tnb"], c["kP"],
               c["jstart"], c["jend"])
    for k in ("Qnew", "Varnew", "Knew", "Gnew"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert a["n_clamped"] == b["n_clamped"]


def test_truncating_row_rule_differs_from_floor():
    """linear_int truncates the offset and the step separately: with a
    26.98 K step the row of T = Tnb[0] + 2 x 26.98 + 1 is 2 (53/26), and a
    temperature up to 1 K below Tnb[0] still maps to row 0 unclamped."""
    Tnb = 300.0 + 26.98 * np.arange(5)
    kP = np.array([1.0, 2.0, 4.0, 8.0, 16.0])
    z = np.zeros((3, 3, 3), np.float32)

    def K(T):
        T1 = np.full((3, 3, 3), T / 1000.0)
        return OD.dns_source(z, z, T1, 1000.0, 1.0, 1.0, 5.67e-08, Tnb, kP, 1, 1)

    r = K(Tnb[0] + 2 * 26.98 + 1.0)
    # int(54.96) / int(26.98) = 54 / 26 = 2: row 2
    x0 = (Tnb[0] + 2 * 26.98 + 1.0) / 1000.0 * 1000.0
    want = (kP[3] - kP[2]) / (Tnb[3] - Tnb[2]) * (x0 - Tnb[2]) + kP[2]
    assert r["Knew"][0, 0, 0] == want and r["n_clamped"] == 0
    r = K(Tnb[0] - 0.9)
    assert r["n_clamped"] == 0 and r["Knew"][0, 0, 0] < kP[0]
    r = K(Tnb[0] - 30.0)
    assert r["n_clamped"] == r["Knew"].size == 3


def test_isothermal_known_answer():
    """T1 on a table row gives Knew = kP there, and Gnew = 4 T1^4 - Qnew/kP."""
    Tnb = 300.0 + 20.0 * np.arange(10)
    kP = np.linspace(0.1, 1.0, 10)
    Q = np.full((4, 4, 5), 3.0e4, np.float32)
    S = np.full((4, 4, 5), 1.0e2, np.float32)
    T1 = np.full((4, 4, 5), 400.0 / 500.0)
    r = OD.dns_source(Q, S, T1, 500.0, 0.5, 1.0, 5.67e-08, Tnb, kP, 1, 2)
    assert np.all(r["Knew"] == kP[5])
    qn = 3.0e4 / 5.67e-08 / 500.0 ** 4
    np.testing.assert_allclose(r["Qnew"][:, :, 1:-1], qn, rtol=1e-15)
    np.testing.assert_allclose(r["Qnew"][:, :, 0], qn / 0.5, rtol=1e-15)
    np.testing.assert_allclose(r["Gnew"][:, :, 1:-1], 4 * 0.8 ** 4 - qn / kP[5], rtol=1e-14)


def test_read_planck_mean_matches_read_kp(tmp_path):
    ts = W.tables_nb(nB=12, nQ=8, nT=16)
    ts.write_dir(tmp_path)
    path = os.path.join(tmp_path, "planck-mean.txt")
    T0, k0 = api.read_planck_mean(path, 16, 0.5)
    T1, k1 = OD.read_kp(path, 16, 0.5)
    np.testing.assert_array_equal(T0, T1)
    np.testing.assert_array_equal(k0, k1)
    a = ts.arrays()
    np.testing.assert_allclose(T0, a["Tnb"], rtol=1e-6)
    np.testing.assert_allclose(k0, 0.5 * a["kP"], rtol=1e-6)
    with pytest.raises(Exception):
        api.read_planck_mean(path, 17, 0.5)


def test_coupling_struct_and_shapes():
    p = W.channel_params(16, 12, 8)
    c = api.DnsCoupling(Tin=955.0, Height=0.5, underrelax=1.0, Tnb=np.arange(4) * 10.0 + 300, kP=np.ones(4),
                        jstart=3, jend=7)
    s = c.struct(p.jmax)
    assert (s.nTemp, s.jstart, s.jend) == (4, 3, 7) and s.Tnb[3] == 330.0 and math.isclose(s.stefan, 5.67e-08)
    assert c.pencil_shapes(p) == ((10, 7, 18), (8, 5, 18))
    c.jend = -1
    assert c.struct(p.jmax).jend == 12
