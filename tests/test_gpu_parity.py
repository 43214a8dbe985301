"""GPU vs CPU oracle parity through the C ABI.

With the same Philox counters the device and the oracle must agree bit for
bit on every sampled band, g point, emission direction, visited cell and
per-bundle FP64 tally, and -- with the same rays_per_thread, which fixes the
FP64 summation order -- on every per-cell mean and variance.
"""
import numpy as np
import pytest

from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    return O


def rand_ids(p, n, seed, kinds=(0,)):
    rng = np.random.default_rng(seed)
    kl = p.kmax // p.p_col
    out = []
    for t in range(n):
        kind = int(kinds[t % len(kinds)])
        out.append((kind, int(rng.integers(1, p.imax + 1)), int(rng.integers(1, p.jmax + 1)),
                    int(rng.integers(1, kl + 1)), int(rng.integers(0, p.nVar)), int(rng.integers(0, p.photmax))))
    return out


def compare_traces(g, gc, o, oc):
    for a, b in zip(g, o):
        assert (a.nb, a.g, a.nsteps, a.end_level) == (b.nb, b.g, b.nsteps, b.end_level)
        assert (a.sx, a.sy, a.sz, a.tra) == (b.sx, b.sy, b.sz, b.tra)
        assert a.De == b.De
    np.testing.assert_array_equal(gc, oc)


def test_trace_parity_grey():
    O = _oracle()
    p = W.config_grey_32(photmax=16, nVar=2)
    T = W.channel_field(p)
    s = api.Solver(p)
    t = s.solve_async(T)
    ids = rand_ids(p, 512, 1)
    g, gc = s.trace(t, ids, max_cells=96)
    o, oc = O.trace(p, None, T, ids, max_cells=96)
    compare_traces(g, gc, o, oc)
    assert sum(r.nsteps for r in g) > 512 * 5
    s.release(t)


def test_trace_parity_narrowband_levels_walls():
    O = _oracle()
    tabs = W.tables_nb()
    p = W.channel_params(32, 32, 32, photmax=32, nVar=2, levels=[(32, 32, 32), (16, 16, 16), (8, 8, 8)],
                         maxs=[5, 5, 100000], calcwalls=1, adiabw=1, adiabe=1)
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    ids = rand_ids(p, 768, 2, kinds=(0, 0, 1, 2))
    g, gc = s.trace(t, ids, max_cells=64)
    o, oc = O.trace(p, tabs, T, ids, max_cells=64)
    compare_traces(g, gc, o, oc)
    assert max(r.end_level for r in g) == 2
    s.release(t)


@pytest.mark.parametrize("bd_y,bd_z", [(3, 4), (5, 2), (4, 3)])
def test_trace_parity_wall_types(bd_y, bd_z):
    O = _oracle()
    tabs = W.tables_nb()
    p = W.channel_params(24, 16, 16, photmax=16, nVar=2, bd_y=bd_y, bd_z=bd_z, adiabw=0, adiabe=1)
    p.Tw[2], p.Tw[3], p.Tw[4], p.Tw[5] = 700.0, 650.0, 800.0, 600.0
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    ids = rand_ids(p, 512, 3)
    g, gc = s.trace(t, ids, max_cells=48)
    o, oc = O.trace(p, tabs, T, ids, max_cells=48)
    compare_traces(g, gc, o, oc)
    s.release(t)


def test_q_parity_grey_32_full():
    """Grey 32^3 (photmax 64, nVar 4): every cell equal to the oracle."""
    O = _oracle()
    p = W.config_grey_32()
    T = W.channel_field(p)
    s = api.Solver(p)
    r = s.solve(T)
    rpt = s.get_launch()[0]
    o = O.solve(p, None, T, rpt=rpt)
    np.testing.assert_array_equal(r.q64, o["q64"])
    np.testing.assert_array_equal(r.var64, o["var64"])
    # Fortran-layout float outputs: interior = Q, sigma = sqrt(var)
    np.testing.assert_array_equal(r.Q[1:-1, 1:-1, 1:-1], o["q64"].astype(np.float32))
    np.testing.assert_array_equal(r.sigma[1:-1, 1:-1, 1:-1], np.sqrt(o["var64"]).astype(np.float32))


def test_q_parity_narrowband_64_subset_and_walls():
    """Narrow-band 64^3, 3 levels, adiabatic west wall with wall flux."""
    O = _oracle()
    tabs = W.tables_nb()
    p = W.config_nb_64(photmax=32)
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    r = s.solve(T)
    rpt = s.get_launch()[0]
    o = O.solve(p, tabs, T, rpt=rpt, cell_begin=0, cell_end=3 * 64 * 64)
    np.testing.assert_array_equal(r.q64[:3], o["q64"][:3])
    np.testing.assert_array_equal(r.var64[:3], o["var64"][:3])
    np.testing.assert_array_equal(r.qw64, o["qw64"])
    np.testing.assert_array_equal(r.vw64, o["vw64"])
    # east wall is not adiabatic: zero in the Fortran array (mc_gpu_noint.cu:996-1001)
    assert np.all(r.Q[1:-1, 1:-1, -1] == 0) and np.all(r.Q[1:-1, 1:-1, 0] != 0)


def test_fp64_build_parity():
    O = _oracle()
    tabs = W.tables_nb(logk_lo=-1.0)
    p = W.channel_params(16, 16, 16, photmax=16, nVar=3, calcwalls=1, adiabw=1, adiabe=1, floatpoint=1)
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    r = s.solve(T)
    o = O.solve(p, tabs, T, rpt=s.get_launch()[0], fp64=True)
    np.testing.assert_array_equal(r.q64, o["q64"])
    np.testing.assert_array_equal(r.qw64, o["qw64"])


def test_launch_knobs_do_not_change_results():
    tabs = W.tables_nb()
    p = W.channel_params(32, 16, 16, photmax=64, nVar=2)
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    s.set_launch(rays_per_thread=8, block_threads=256)
    a = s.solve(T)
    s.set_launch(rays_per_thread=8, block_threads=128)
    b = s.solve(T)
    np.testing.assert_array_equal(a.q64, b.q64)  # same summation order
    s.set_launch(rays_per_thread=8, block_threads=256, occupancy=4)
    np.testing.assert_array_equal(s.solve(T).q64, a.q64)
    s.set_launch(rays_per_thread=32, block_threads=128, occupancy=2)
    c = s.solve(T)
    np.testing.assert_allclose(c.q64, a.q64, rtol=1e-11, atol=1e-9 * np.abs(a.q64).max())


def test_batch_equals_alone():
    probs = W.batch_problems(n=6, seed=5, edges=(8, 12, 16), photmaxes=(16, 32))
    solvers, fields, alone = [], [], []
    for pr in probs:
        tabs = None if pr["grey"] else W.tables_nb(nB=pr["nB"], seed=pr["table_seed"])
        s = api.Solver(pr["params"], tabs)
        T = W.channel_field(pr["params"], seed=pr["field_seed"])
        solvers.append((s, tabs))
        fields.append(T)
        alone.append(s.solve(T))
    for use_graph in (False, True):
        b = api.Batch(use_graph=use_graph)
        for (s, _), T in zip(solvers, fields):
            b.add(s, T)
        for rep in range(2):
            b.run()
            b.wait()
            for i in range(len(probs)):
                r = b.collect(i)
                np.testing.assert_array_equal(r.q64, alone[i].q64)
                np.testing.assert_array_equal(r.Q, alone[i].Q)
        b.close()


def test_legacy_entry_points_match_solver():
    import ctypes as C
    from radchan_b200 import _lib as L
    tabs = W.tables_nb()
    p = W.channel_params(16, 16, 16, photmax=32, nVar=2, calcwalls=1, adiabw=1, adiabe=1)
    T = W.channel_field(p)
    ref = api.Solver(p, tabs).solve(T)
    L.check(L.lib().rc_legacy_configure(C.byref(p), C.byref(tabs.view)))
    Q = np.full(api.result_shape(p), -7.0, np.float32)
    S = np.full(api.result_shape(p), -7.0, np.float32)
    z = C.c_int(1)
    rank = C.c_int(0)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    L.lib().mc_gpu_(fp(T), C.byref(z), C.byref(rank))
    L.lib().get_results_(fp(Q), fp(S), C.byref(rank))
    L.lib().rc_legacy_release()
    np.testing.assert_array_equal(Q[1:-1, 1:-1, :], ref.Q[1:-1, 1:-1, :])
    np.testing.assert_array_equal(S[1:-1, 1:-1, :], ref.sigma[1:-1, 1:-1, :])
    # ghost layers other than the wall columns are left untouched
    assert np.all(Q[0] == -7.0) and np.all(Q[:, 0] == -7.0)


def test_nonfinite_temperature_is_reported():
    p = W.config_grey_32(photmax=4, nVar=2)
    T = W.channel_field(p)
    T[5, 5, 5] = np.nan
    s = api.Solver(p)
    t = s.solve_async(T)
    info = s.info(t)
    assert info.status & 2
    with pytest.raises(Exception):
        s.collect(t)


def test_solve_info_counts():
    p = W.config_grey_32(photmax=8, nVar=2)
    T = W.channel_field(p)
    s = api.Solver(p)
    t = s.solve_async(T)
    info = s.info(t)
    assert info.bundles == 32 ** 3 * 2 * 8
    assert info.steps > info.bundles
    assert info.status == 0
    O = _oracle()
    su = O.setup(p, None, T)
    assert info.Tmax == su.Tmax and info.table_row == su.row
    s.release(t)
