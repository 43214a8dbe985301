"""Particle scattering on the device against the CPU oracle, through the C ABI.

The scattering variant of the march draws every event from the bundle's own
Philox counter, so with the same rays_per_thread the device and the oracle
agree bit for bit on traces (band, g point, every visited cell including
the cells of scattering events, final transmissivity, tally) and on every
per-cell mean, variance and wall flux.  Covered: grey gas with forward
scattering, narrow band with multigrid levels and both wall fluxes,
specular y walls, the FP64 build, a batch that mixes a scattering and a
non-scattering problem, removing the scattering again, and served requests
with particles per table set.
"""
import numpy as np
import pytest

from radchan_b200 import api
from radchan_b200 import workloads as W

from phase_tables import odd_phase_cdfs

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    return O


def _equal(r, o):
    for key in ("q64", "var64", "qw64", "vw64"):
        assert np.array_equal(getattr(r, key), o[key]), key


def _nb_case(photmax=16, **kw):
    tabs = W.tables_nb(nB=24, nQ=4, nT=32)
    p = W.channel_params(16, 8, 8, photmax=photmax, nVar=2, nB=24, nQ=4, nT=32, levels=[(16, 8, 8), (8, 4, 4)],
                         maxs=[5, 100000], calcwalls=1, adiabw=1, adiabe=1, **kw)
    sc = api.Scattering.synthetic(nB=24, nQ=4, nA=91, ksca_lo=0.2, ksca_hi=6.0, g_lo=-0.4, g_hi=0.9, seed=13)
    return p, tabs, sc


def test_grey_forward_scattering_equals_oracle():
    O = _oracle()
    p = W.channel_params(16, 16, 16, grey=True, photmax=32, nVar=2)
    sc = api.Scattering.synthetic(nB=p.grey_nB, nQ=1, nA=181, ksca_lo=1.5, ksca_hi=1.5, g_lo=0.6, g_hi=0.6)
    T = W.channel_field(p, seed=5)
    s = api.Solver(p)
    s.set_scattering(sc)
    t = s.solve_async(T)
    info = s.info(t)
    r = s.collect(t)
    o = O.solve(p, None, T, rpt=s.get_launch()[0], scatter=sc.arrays())
    _equal(r, o)
    assert info.steps == o["steps"]
    s.close()


@pytest.mark.parametrize("bd_y", [1, 3])
def test_narrowband_levels_walls_scattering_equals_oracle(bd_y):
    O = _oracle()
    p, tabs, sc = _nb_case(bd_y=bd_y)
    T = W.channel_field(p, seed=6)
    s = api.Solver(p, tabs)
    s.set_scattering(sc)
    r = s.solve(T)
    o = O.solve(p, tabs, T, rpt=s.get_launch()[0], scatter=sc.arrays())
    _equal(r, o)
    assert np.any(r.qw64 != 0)
    s.close()


def test_scattering_traces_equal_oracle():
    O = _oracle()
    p, tabs, sc = _nb_case(photmax=32)
    T = W.channel_field(p, seed=7)
    s = api.Solver(p, tabs)
    s.set_scattering(sc)
    t = s.solve_async(T)
    rng = np.random.default_rng(2)
    ids = []
    for n in range(400):
        kind = n % 3
        ids.append((kind, int(rng.integers(1, p.imax + 1)), int(rng.integers(1, p.jmax + 1)),
                    int(rng.integers(1, p.kmax + 1)), int(rng.integers(0, p.nVar)), int(rng.integers(0, p.photmax))))
    g, gc = s.trace(t, ids, max_cells=128)
    o, oc = O.trace(p, tabs, T, ids, max_cells=128, scatter=sc.arrays())
    for a, b in zip(g, o):
        assert (a.nb, a.g, a.nsteps, a.end_level) == (b.nb, b.g, b.nsteps, b.end_level)
        assert (a.sx, a.sy, a.sz, a.tra) == (b.sx, b.sy, b.sz, b.tra)
        assert a.De == b.De
    np.testing.assert_array_equal(gc, oc)
    # scattering events appear as repeated cells: some bundle visits the same
    # cell on two consecutive steps
    rep = (gc[:, 1:, :] == gc[:, :-1, :]).all(axis=2) & (gc[:, 1:, 0] >= 0)
    assert rep.any()
    s.release(t)
    s.close()


def test_fp64_build_with_scattering_equals_fp64_oracle():
    O = _oracle()
    p, tabs, sc = _nb_case(photmax=8, floatpoint=1)
    T = W.channel_field(p, seed=8)
    s = api.Solver(p, tabs)
    s.set_scattering(sc)
    r = s.solve(T)
    o = O.solve(p, tabs, T, rpt=s.get_launch()[0], fp64=True, scatter=sc.arrays())
    _equal(r, o)
    s.close()


def test_batch_mixing_scattering_and_plain_problems_equals_alone():
    p1, tabs, sc = _nb_case(photmax=16)
    p2 = W.channel_params(12, 8, 8, grey=True, photmax=32, nVar=2)
    T1 = W.channel_field(p1, seed=9)
    T2 = W.channel_field(p2, seed=10)
    s1 = api.Solver(p1, tabs)
    s1.set_scattering(sc)
    s2 = api.Solver(p2)
    alone1, alone2 = s1.solve(T1), s2.solve(T2)
    b = api.Batch(use_graph=True)
    b.add(s1, T1)
    b.add(s2, T2)
    b.run()
    b.wait()
    r1, r2 = b.collect(0), b.collect(1)
    _equal(r1, dict(q64=alone1.q64, var64=alone1.var64, qw64=alone1.qw64, vw64=alone1.vw64))
    _equal(r2, dict(q64=alone2.q64, var64=alone2.var64, qw64=alone2.qw64, vw64=alone2.vw64))
    b.close()
    s1.close()
    s2.close()


def test_removing_scattering_restores_the_plain_solve():
    p, tabs, sc = _nb_case(photmax=16)
    T = W.channel_field(p, seed=11)
    s = api.Solver(p, tabs)
    plain = s.solve(T)
    s.set_scattering(sc)
    scat = s.solve(T)
    s.set_scattering(None)
    again = s.solve(T)
    assert not np.array_equal(plain.q64, scat.q64)
    _equal(again, dict(q64=plain.q64, var64=plain.var64, qw64=plain.qw64, vw64=plain.vw64))
    s.close()


def test_scattering_table_mismatch_is_rejected():
    p, tabs, _ = _nb_case()
    s = api.Solver(p, tabs)
    wrong = api.Scattering.synthetic(nB=20, nQ=4, nA=31)
    with pytest.raises(RuntimeError):
        s.set_scattering(wrong)
    s.close()


def test_served_requests_with_particles_equal_alone():
    """The server takes particles per table set (and for grey requests):
    requests solved in the mix equal the same solves alone, bit for bit; a
    request submitted after the particles are removed solves without them
    while the earlier ones keep theirs."""
    p1, tabs, sc = _nb_case(photmax=32)
    pg = W.channel_params(12, 8, 8, grey=True, photmax=32, nVar=2)
    scg = api.Scattering.synthetic(nB=pg.grey_nB, nQ=1, nA=91, ksca_lo=0.8, ksca_hi=0.8, g_lo=0.5, g_hi=0.5)
    T1, Tg = W.channel_field(p1, seed=21), W.channel_field(pg, seed=22)
    s = api.Solver(p1, tabs)
    plain = s.solve(T1, want64=False)
    s.set_scattering(sc)
    scat = s.solve(T1, want64=False)
    s.close()
    s = api.Solver(pg)
    s.set_scattering(scg)
    grey = s.solve(Tg, want64=False)
    s.close()
    assert not np.array_equal(plain.Q, scat.Q)
    srv = api.Server(max_inflight=8)
    ts = srv.add_tables(tabs)
    srv.set_scattering(ts, sc)
    srv.set_scattering(-1, scg)
    a = srv.submit(p1, T1, table_set=ts)
    g = srv.submit(pg, Tg)
    srv.set_scattering(ts, None)
    b = srv.submit(p1, T1, table_set=ts)
    ra, rg, rb = srv.wait(a), srv.wait(g), srv.wait(b)
    srv.close()
    np.testing.assert_array_equal(ra.Q, scat.Q)
    np.testing.assert_array_equal(ra.sigma, scat.sigma)
    np.testing.assert_array_equal(rg.Q, grey.Q)
    np.testing.assert_array_equal(rb.Q, plain.Q)


def test_batch_follows_a_member_changed_after_capture():
    """A batch captured into a CUDA graph is captured again when a member's
    particles or launch knobs change afterwards (its descriptors would be
    stale): each run equals the member solved alone as it is then."""
    p1, tabs, sc = _nb_case(photmax=16)
    T1 = W.channel_field(p1, seed=31)

    def alone(scatter, rpt):
        s = api.Solver(p1, tabs)
        if scatter:
            s.set_scattering(sc)
        s.set_launch(rays_per_thread=rpt)
        r = s.solve(T1)
        s.close()
        return r

    s1 = api.Solver(p1, tabs)
    rpt0 = s1.get_launch()[0]
    b = api.Batch(use_graph=True)
    b.add(s1, T1)
    results = []
    for change in (None, "particles", "knobs"):
        if change == "particles":
            s1.set_scattering(sc)
        elif change == "knobs":
            s1.set_launch(rays_per_thread=2 * rpt0)
        b.run()
        b.wait()
        results.append(b.collect(0))
    b.close()
    s1.close()
    for r, (scatter, rpt) in zip(results, ((False, rpt0), (True, rpt0), (True, 2 * rpt0))):
        a = alone(scatter, rpt)
        _equal(r, dict(q64=a.q64, var64=a.var64, qw64=a.qw64, vw64=a.vw64))


def test_phase_cdf_with_flat_runs_and_jumps_equals_oracle():
    """The device finds a scattering angle by a bracketed search of the
    band's phase CDF (a guide per band); the oracle bisects the whole table.
    On CDFs with flat stretches, jumps and long tails both pick the same
    angle: traces and results agree bit for bit."""
    O = _oracle()
    p, tabs, _ = _nb_case(photmax=32)
    nA = 91
    theta = np.linspace(0.0, np.pi, nA)
    rng = np.random.default_rng(4)
    sc = api.Scattering.from_arrays(rng.uniform(1.0, 6.0, (24, 4)), theta, odd_phase_cdfs(24, nA, 5))
    assert sc.validate() == ""
    T = W.channel_field(p, seed=12)
    s = api.Solver(p, tabs)
    s.set_scattering(sc)
    t = s.solve_async(T)
    ids = [(k % 3, 1 + k % p.imax, 1 + (k // 3) % p.jmax, 1 + (k // 7) % p.kmax, k % p.nVar, k % p.photmax)
           for k in range(300)]
    g, gc = s.trace(t, ids, max_cells=128)
    o, oc = O.trace(p, tabs, T, ids, max_cells=128, scatter=sc.arrays())
    for a, b in zip(g, o):
        assert (a.nb, a.g, a.nsteps, a.sx, a.sy, a.sz, a.tra) == (b.nb, b.g, b.nsteps, b.sx, b.sy, b.sz, b.tra)
    np.testing.assert_array_equal(gc, oc)
    r = s.collect(t)
    _equal(r, O.solve(p, tabs, T, rpt=s.get_launch()[0], scatter=sc.arrays()))
    s.close()
