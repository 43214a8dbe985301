"""DNS coupling on the GPU (rc_dns_source, rc_dns_source_device,
rc_legacy_source): the fused kernel equals the CPU restatement of
GET_RESULTS + fix_rad + fix_kappa + the Gnew loop bit for bit, on the
device and host entry points; the DNS's lagged launch pattern
(src/dns/channel.f:237-256) gives the same answers as synchronous solves."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from oracle import dns as OD
from radchan_b200 import _lib as L
from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu

TIN = 955.0


def _problem(jstart=1, jend=-1, seed=3, **kw):
    tabs = W.tables_nb(nB=40, nQ=4, nT=32)
    p = W.channel_params(32, 16, 16, photmax=16, nVar=4, nB=40, nQ=4, nT=32,
                         levels=[(32, 16, 16), (16, 8, 8)], maxs=[5, 100000], calcwalls=1, adiabw=1, **kw)
    a = tabs.arrays()
    Tnb, kP = a["Tnb"].astype(np.float64), a["kP"].astype(np.float64) * 0.5
    cpl = api.DnsCoupling(Tin=TIN, Height=0.5, underrelax=0.8, Tnb=Tnb, kP=kP, jstart=jstart, jend=jend)
    T1 = W.channel_field(p, seed=seed).astype(np.float64) / TIN
    return p, tabs, cpl, T1


def _pencil(T1, cpl, p):
    je = p.jmax if cpl.jend < 0 else cpl.jend
    return np.ascontiguousarray(T1[:, cpl.jstart - 1:je + 2, :])


def _oracle(r, T1p, cpl, p):
    je = p.jmax if cpl.jend < 0 else cpl.jend
    return OD.dns_source(r.Q, r.sigma, T1p, cpl.Tin, cpl.Height, cpl.underrelax, cpl.stefan, cpl.Tnb, cpl.kP,
                         cpl.jstart, je)


def _equal(a, b):
    for k in ("Qnew", "Varnew", "Knew", "Gnew"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert a["n_clamped"] == b["n_clamped"]


@pytest.mark.parametrize("jstart,jend,adiabe", [(1, -1, 0), (5, 12, 1), (16, 16, 1)])
def test_device_and_host_entry_points_equal_oracle(jstart, jend, adiabe):
    import torch
    p, tabs, cpl, T1 = _problem(jstart, jend, adiabe=adiabe)
    T = api.field_from_dns(T1, TIN)
    T1p = _pencil(T1, cpl, p)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    _, oshape = cpl.pencil_shapes(p)
    dev = torch.device("cuda:0")
    T1d = torch.from_numpy(T1p).to(dev)
    outs = [torch.full(oshape, np.nan, dtype=torch.float64, device=dev) for _ in range(4)]
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    # a stream of the caller's: the kernel waits for the solve on it
    side = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    s.dns_source_device(t, cpl, T1d.data_ptr(), *[o.data_ptr() for o in outs], cnt.data_ptr(),
                        stream=side.cuda_stream)
    side.synchronize()
    r = s.collect(t)
    want = _oracle(r, T1p, cpl, p)
    got = dict(zip(("Qnew", "Varnew", "Knew", "Gnew"), (o.cpu().numpy() for o in outs)))
    got["n_clamped"] = int(cnt.item())
    _equal(got, want)
    # walls: west flux computed, east only when adiabatic
    assert np.all(want["Qnew"][:, :, 0] != 0)
    assert np.all(want["Qnew"][:, :, -1] == 0) == (not adiabe)
    # the host entry point on a second, identical solve
    h = s.dns_source(s.solve_async(T), cpl, T1p)
    _equal(h, want)
    s.close()


def test_rows_outside_the_table_are_extended_and_counted():
    p, tabs, cpl, T1 = _problem()
    T = api.field_from_dns(T1, TIN)
    T1p = _pencil(T1, cpl, p).copy()
    Tnb0, step = cpl.Tnb[0], cpl.Tnb[1] - cpl.Tnb[0]
    # int(x0 - Tnb[0]) / int(step) truncates toward zero: up to one step
    # below Tnb[0] still maps to row 0, two steps below does not
    T1p[2, 4, 5] = (Tnb0 - 0.9 * step) / TIN
    T1p[3, 4, 5] = (Tnb0 - 2.0 * step) / TIN
    T1p[4, 6, 7] = 2500.0 / TIN     # above the last row
    s = api.Solver(p, tabs)
    r = s.solve(T)
    h = s.dns_source(s.solve_async(T), cpl, T1p)
    want = _oracle(r, T1p, cpl, p)
    _equal(h, want)
    assert h["n_clamped"] == 2
    s.close()


def test_lagged_launch_pattern_equals_synchronous_solves():
    """channel.f:237-256: MC_GPU at istart, then every radStep steps
    GET_RESULTS of the previous launch and a new MC_GPU on the current
    field; also with the next launch issued before the previous is read
    (two slots: the fields are double-buffered)."""
    p, tabs, cpl, _ = _problem()
    fields = [W.channel_field(p, seed=40 + n).astype(np.float64) / TIN for n in range(4)]
    ref = api.Solver(p, tabs)
    want = [_oracle(ref.solve(api.field_from_dns(f, TIN)), _pencil(f, cpl, p), cpl, p) for f in fields[:3]]
    s = api.Solver(p, tabs)
    t = s.solve_async(api.field_from_dns(fields[0], TIN))
    for n in range(1, 4):
        got = s.dns_source(t, cpl, _pencil(fields[n - 1], cpl, p))
        t = s.solve_async(api.field_from_dns(fields[n], TIN))
        _equal(got, want[n - 1])
    s.release(t)
    t = s.solve_async(api.field_from_dns(fields[0], TIN))
    for n in range(1, 4):
        t_next = s.solve_async(api.field_from_dns(fields[n], TIN))
        got = s.dns_source(t, cpl, _pencil(fields[n - 1], cpl, p))
        _equal(got, want[n - 1])
        t = t_next
    s.release(t)
    s.close()
    ref.close()


def test_legacy_source_matches_solver():
    p, tabs, cpl, T1 = _problem(4, 9)
    T = api.field_from_dns(T1, TIN)
    T1p = _pencil(T1, cpl, p)
    s = api.Solver(p, tabs)
    want = s.dns_source(s.solve_async(T), cpl, T1p)
    s.close()
    L.check(L.lib().rc_legacy_configure(C.byref(p), C.byref(tabs.view)))
    z, rank = C.c_int(1), C.c_int(0)
    L.lib().mc_gpu_(T.ctypes.data_as(C.POINTER(C.c_float)), C.byref(z), C.byref(rank))
    _, oshape = cpl.pencil_shapes(p)
    out = {k: np.empty(oshape) for k in ("Qnew", "Varnew", "Knew", "Gnew")}
    n = C.c_longlong()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    st = cpl.struct(p.jmax)
    L.check(L.lib().rc_legacy_source(C.byref(st), dp(T1p), dp(out["Qnew"]), dp(out["Varnew"]), dp(out["Knew"]),
                                      dp(out["Gnew"]), C.byref(n)))
    out["n_clamped"] = n.value
    # nothing pending any more
    assert L.lib().rc_legacy_source(C.byref(st), dp(T1p), dp(out["Qnew"]), dp(out["Varnew"]), dp(out["Knew"]),
                                    dp(out["Gnew"]), None) == -5
    L.lib().rc_legacy_release()
    _equal(out, want)


def test_coupling_validation():
    p, tabs, cpl, T1 = _problem()
    T = api.field_from_dns(T1, TIN)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    T1p = _pencil(T1, cpl, p)
    for bad in (dict(jstart=0), dict(jend=p.jmax + 1), dict(Tnb=cpl.Tnb[:1], kP=cpl.kP[:1]),
                dict(Tnb=300.0 + 0.5 * np.arange(len(cpl.Tnb))), dict(Tin=0.0)):
        c2 = dataclasses.replace(cpl, **bad)
        T1b = np.zeros(c2.pencil_shapes(p)[0]) if ("jstart" in bad or "jend" in bad) else T1p
        with pytest.raises(L.RadChanError) as e:
            s.dns_source(t, c2, T1b)
        assert e.value.code == -1
    # the ticket survived the refused calls
    h = s.dns_source(t, cpl, T1p)
    assert np.isfinite(h["Gnew"]).all()
    s.close()
