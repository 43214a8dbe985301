"""Edge cases of the solve path, bit for bit against the oracle: z-slabs of
a multi-slab decomposition (p_col > 1, zstart > 1, mc_gpu_noint.cu:97), odd
grid extents with a zero-width centre cell, one cell across a dimension,
photmax 1, two replicates, temperatures outside the table range, and
argument checks that fail before any launch."""
import numpy as np
import pytest

from radchan_b200 import _lib as L
from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _oracle():
    from oracle import oracle as O
    return O


def _same(p, tabs, T, zstart=1):
    O = _oracle()
    s = api.Solver(p, tabs)
    t = s.solve_async(T, zstart=zstart)
    r = s.collect(t)
    o = O.solve(p, tabs, T, zstart=zstart, rpt=s.get_launch()[0])
    np.testing.assert_array_equal(r.q64, o["q64"])
    np.testing.assert_array_equal(r.var64, o["var64"])
    np.testing.assert_array_equal(r.qw64, o["qw64"])
    np.testing.assert_array_equal(r.vw64, o["vw64"])
    s.close()
    return r


@pytest.mark.parametrize("zstart", [1, 9, 25])
def test_z_slab_of_a_multi_slab_decomposition(zstart):
    tabs = W.tables_nb(nB=30, nQ=4, nT=32)
    p = W.channel_params(24, 16, 32, photmax=32, nVar=2, nB=30, nQ=4, nT=32, calcwalls=1, adiabw=1, adiabe=1,
                         levels=[(24, 16, 32), (12, 8, 16)], maxs=[5, 100000])
    p.p_col = 4                      # kloc = 8 planes per slab
    T = W.channel_field(p, seed=zstart)
    r = _same(p, tabs, T, zstart=zstart)
    assert r.q64.shape == (8, 16, 24)


def test_odd_extents_and_single_cell_dimension():
    p = W.channel_params(17, 9, 1, grey=True, photmax=16, nVar=2)
    _same(p, None, W.channel_field(p, seed=2))


def test_photmax_one_and_two_replicates():
    tabs = W.tables_nb(nB=20, nQ=8, nT=16)
    p = W.channel_params(12, 8, 8, photmax=1, nVar=2, nB=20, nQ=8, nT=16, calcwalls=1, adiabw=1)
    _same(p, tabs, W.channel_field(p, seed=3))


def test_temperatures_outside_the_table_are_clamped_and_flagged():
    tabs = W.tables_nb(nB=20, nQ=4, nT=16)   # tables cover 300..2000 K
    p = W.channel_params(12, 8, 8, photmax=8, nVar=2, nB=20, nQ=4, nT=16)
    T = W.channel_field(p, seed=4)
    T[3, 3, 3:6] = 250.0                     # below the first table row
    _same(p, tabs, T)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    assert s.info(t).status & 1
    s.release(t)


def test_bad_arguments_fail_before_launch():
    p = W.config_grey_32(photmax=4, nVar=2)
    s = api.Solver(p)
    T = W.channel_field(p)
    with pytest.raises(AssertionError):
        s.solve_async(T[:, :, :-1])                      # wrong field shape
    with pytest.raises(L.RadChanError):
        s.solve_async(T, zstart=2)                       # slab beyond kmax
    q = api.copy_params(p)
    q.nVar = 0
    with pytest.raises(L.RadChanError):
        api.Solver(q)
    s.close()


@pytest.mark.parametrize("grey", [False, True])
def test_band_and_g_search_edges_equal_the_oracle(grey):
    """The device's band / g-point searches (select_band_g, used by every
    emission) against the oracle on uniforms placed on, just below and just
    above every CDF entry, at 0, just below 1 and at 1; the oracle follows
    the reference's bisection rule on the same uniforms
    (tests/test_cpu_band_search.py)."""
    from test_cpu_band_search import _problem, edge_uniforms
    O = _oracle()
    p, tabs, T = _problem(grey)
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    _, _, cdf_f, cdf_s, probq, row = O.sample_bands(p, tabs, T, 0, [0.5], [0.5])
    cases = [(0, edge_uniforms(cdf_f), None)]
    cases.append((1, np.unique(np.concatenate([edge_uniforms(cdf_s), edge_uniforms(cdf_f[:1], n_random=0)])), None))
    if not grey:
        a = tabs.arrays()
        for b in (0, 7, 39):
            ub = np.float32(np.nextafter(cdf_f[b], np.float32(0)))
            ug = edge_uniforms(a["probg"][row, b], seed=b, n_random=50)
            cases.append((0, np.full_like(ug, ub), ug))
        cases.append((2, np.full(60, 0.5, np.float32), edge_uniforms(probq, n_random=50)[:60]))
    for kind, ub, ug in cases:
        if ug is None:
            ug = np.full_like(ub, 0.5)
        n = min(ub.size, ug.size)
        ub, ug = ub[:n], ug[:n]
        nb_d, g_d = s.sample_bands(t, kind, ub, ug)
        nb_o, g_o, _, _, _, _ = O.sample_bands(p, tabs, T, kind, ub, ug)
        assert np.array_equal(nb_d, nb_o), kind
        assert np.array_equal(g_d, g_o), kind
    s.release(t)
    s.close()
