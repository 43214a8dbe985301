"""Failure handling without a device fault: host-side injected failures
(rc_debug_fail_next) at every site surface as RC_E_CUDA naming the site,
and the context or server keeps working -- the next solve equals the oracle
or the same request solved alone, bit for bit.  Served requests can be
cancelled while queued or while running."""
import time

import numpy as np
import pytest

from radchan_b200 import _lib as L
from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def _arm(site, n=1):
    L.check(L.lib().rc_debug_fail_next(site.encode(), n))


@pytest.fixture(autouse=True)
def _disarm():
    yield
    for s in ("field_copy", "march", "tally", "collect", "dns", "quantum"):
        L.lib().rc_debug_fail_next(s.encode(), 0)


def _nb():
    tabs = W.tables_nb(nB=24, nQ=4, nT=32)
    p = W.channel_params(16, 8, 8, photmax=16, nVar=2, nB=24, nQ=4, nT=32, levels=[(16, 8, 8), (8, 4, 4)],
                         maxs=[5, 100000], calcwalls=1, adiabw=1)
    return p, tabs, W.channel_field(p, seed=4)


@pytest.mark.parametrize("site", ["field_copy", "march", "tally"])
def test_failed_launch_leaves_the_context_usable(site):
    from oracle import oracle as O
    p, tabs, T = _nb()
    s = api.Solver(p, tabs)
    _arm(site)
    with pytest.raises(L.RadChanError) as e:
        s.solve_async(T)
    assert e.value.code == -2 and ("injected failure at " + site) in str(e.value)
    # both slots are free again: two solves in flight, then the results
    t1, t2 = s.solve_async(T), s.solve_async(T)
    r1, r2 = s.collect(t1), s.collect(t2)
    o = O.solve(p, tabs, T, rpt=s.get_launch()[0])
    np.testing.assert_array_equal(r1.q64, o["q64"])
    np.testing.assert_array_equal(r2.q64, o["q64"])
    np.testing.assert_array_equal(r1.qw64, o["qw64"])
    s.close()


def test_failed_collect_consumes_the_ticket_and_recovers():
    p, tabs, T = _nb()
    s = api.Solver(p, tabs)
    ref = s.solve(T)
    t = s.solve_async(T)
    _arm("collect")
    with pytest.raises(L.RadChanError) as e:
        s.collect(t)
    assert "injected failure at collect" in str(e.value)
    with pytest.raises(L.RadChanError) as e:
        s.collect(t)
    assert e.value.code == -5
    np.testing.assert_array_equal(s.solve(T).q64, ref.q64)
    s.close()


def test_failed_dns_launch_keeps_the_ticket():
    from oracle import dns as OD
    p, tabs, T = _nb()
    a = tabs.arrays()
    cpl = api.DnsCoupling(Tin=955.0, Height=0.5, underrelax=1.0, Tnb=a["Tnb"].astype(np.float64),
                          kP=a["kP"].astype(np.float64) * 0.5)
    T1 = T.astype(np.float64) / 955.0
    Tf = api.field_from_dns(T1, 955.0)
    s = api.Solver(p, tabs)
    r = s.solve(Tf)
    t = s.solve_async(Tf)
    _arm("dns")
    with pytest.raises(L.RadChanError) as e:
        s.dns_source(t, cpl, T1)
    assert "injected failure at dns" in str(e.value)
    h = s.dns_source(t, cpl, T1)
    want = OD.dns_source(r.Q, r.sigma, T1, 955.0, 0.5, 1.0, cpl.stefan, cpl.Tnb, cpl.kP, 1, p.jmax)
    for k in ("Qnew", "Varnew", "Knew", "Gnew"):
        np.testing.assert_array_equal(h[k], want[k])
    s.close()


def test_failed_server_quantum_fails_its_requests_only():
    p, tabs, T = _nb()
    alone = api.Solver(p, tabs).solve(T, want64=False)
    srv = api.Server()
    ts = srv.add_tables(tabs)
    srv.wait(srv.submit(p, T, table_set=ts))   # warm the class
    _arm("quantum")
    a = srv.submit(p, T, table_set=ts)
    with pytest.raises(L.RadChanError) as e:
        srv.wait(a)
    assert e.value.code == -2 and "injected failure at quantum" in str(e.value)
    for _ in range(2):
        r = srv.wait(srv.submit(p, T, table_set=ts))
        np.testing.assert_array_equal(r.Q, alone.Q)
        np.testing.assert_array_equal(r.sigma, alone.sigma)
    srv.close()


def test_cancel_queued_and_running_requests():
    tabs = W.tables_nb(nB=40, nQ=4, nT=32)
    big = W.channel_params(64, 64, 64, photmax=4096, nVar=4, nB=40, nQ=4, nT=32)
    small = W.channel_params(16, 8, 8, photmax=16, nVar=4, nB=40, nQ=4, nT=32)
    Tb, Ts = W.channel_field(big, seed=1), W.channel_field(small, seed=2)
    alone = api.Solver(small, tabs).solve(Ts, want64=False)
    srv = api.Server(max_inflight=1)
    ts = srv.add_tables(tabs)
    srv.wait(srv.submit(small, Ts, table_set=ts))
    a = srv.submit(big, Tb, table_set=ts)     # runs for seconds
    b = srv.submit(small, Ts, table_set=ts)   # queued behind it (max_inflight 1)
    c = srv.submit(small, Ts, table_set=ts)
    srv.cancel(b)
    with pytest.raises(L.RadChanError) as e:
        srv.wait(b)
    assert e.value.code == -9
    time.sleep(0.2)
    t0 = time.perf_counter()
    srv.cancel(a)
    with pytest.raises(L.RadChanError) as e:
        srv.wait(a)
    assert e.value.code == -9
    assert time.perf_counter() - t0 < 5.0
    # the request behind the cancelled ones runs and equals the solve alone
    r = srv.wait(c)
    np.testing.assert_array_equal(r.Q, alone.Q)
    np.testing.assert_array_equal(r.sigma, alone.sigma)
    # the cancelled request's context went back to the pool: its class runs
    q = api.copy_params(big)
    q.photmax = 16
    srv.wait(srv.submit(q, Tb, table_set=ts))
    with pytest.raises(L.RadChanError) as e:
        srv.cancel(a)                          # already waited
    assert e.value.code == -8
    # a cancel racing the end of a short solve: either outcome is whole
    d = srv.submit(small, Ts, table_set=ts)
    try:
        srv.cancel(d)
        accepted = True
    except L.RadChanError as ex:
        assert ex.code == -5                   # already finished: the result stands
        accepted = False
    try:
        np.testing.assert_array_equal(srv.wait(d).Q, alone.Q)
    except L.RadChanError as ex:
        assert accepted and ex.code == -9
    srv.close()
