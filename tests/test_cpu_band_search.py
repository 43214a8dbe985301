"""Edge rules of the band and g-point searches (find_band / find_bandS,
mc_gpu_noint.cu:1103-1233): the oracle against a line-by-line restatement
of the reference's bisection, on uniforms placed exactly on, just below
and just above every CDF entry, at 0, the smallest float, just below 1 and
at 1 (the reference's R == 1 -> last rule; cuRAND's uniforms include 1.0).
The device is checked against the oracle on the same uniforms in
tests/test_gpu_edges.py."""
import numpy as np
import pytest

from oracle import oracle as O
from radchan_b200 import workloads as W


def ref_bisect(cdf, u, edge0=None):
    """The reference's search (mc_gpu_noint.cu:1113-1127): bisection for the
    largest d with R >= cdf[d], plus one; R < cdf[0] -> 0 (find_bandS tests
    the fluid CDF's first entry instead, :1189, :1208 -- edge0); R == 1 ->
    n - 1.  Comparisons in float32, as on the device."""
    cdf = np.asarray(cdf, np.float32)
    u = np.float32(u)
    n = cdf.size
    lo, w = 0, n
    while w > lo + 1:
        d = (lo + w) // 2
        if u < cdf[d]:
            w = d
        if u >= cdf[d]:
            lo = d
    lo += 1
    if u < (cdf[0] if edge0 is None else np.float32(edge0)):
        lo = 0
    if u == np.float32(1):
        lo = n - 1
    return lo


def edge_uniforms(cdf, seed=0, n_random=500):
    """Every CDF entry, its float neighbours, 0, the smallest float, just
    below 1, 1, and seeded random uniforms; all within [0, 1]."""
    c = np.asarray(cdf, np.float32)
    vals = [c, np.nextafter(c, np.float32(0)), np.nextafter(c, np.float32(2))]
    special = np.array([0.0, np.nextafter(np.float32(0), np.float32(1)), np.nextafter(np.float32(1), np.float32(0)),
                        1.0], np.float32)
    rnd = np.random.default_rng(seed).random(n_random).astype(np.float32)
    u = np.concatenate(vals + [special, rnd]).astype(np.float32)
    return np.unique(u[(u >= 0) & (u <= 1)])


def _problem(grey):
    if grey:
        p = W.channel_params(16, 8, 8, grey=True, photmax=4, nVar=2, calcwalls=1, adiabw=1, adiabe=1)
        return p, None, W.channel_field(p, seed=5)
    tabs = W.tables_nb(nB=40, nQ=8, nT=32)
    p = W.channel_params(16, 8, 8, photmax=4, nVar=2, nB=40, nQ=8, nT=32, calcwalls=1, adiabw=1, adiabe=1)
    return p, tabs, W.channel_field(p, seed=5)


@pytest.mark.parametrize("grey", [False, True])
def test_fluid_band_search_follows_the_reference_rule(grey):
    p, tabs, T = _problem(grey)
    _, _, cdf_f, _, _, _ = O.sample_bands(p, tabs, T, 0, [0.5], [0.5])
    u = edge_uniforms(cdf_f)
    nb, _, _, _, _, _ = O.sample_bands(p, tabs, T, 0, u, np.full_like(u, 0.5))
    want = [ref_bisect(cdf_f, x) for x in u]
    assert np.array_equal(nb, want)
    # the edge cases are present
    assert (nb == 0).any() and (nb == cdf_f.size - 1).any() and (u == 1).any()


def test_fluid_g_search_follows_the_reference_rule():
    p, tabs, T = _problem(False)
    a = tabs.arrays()
    _, _, cdf_f, _, _, row = O.sample_bands(p, tabs, T, 0, [0.5], [0.5])
    for b in (0, 7, 39):
        # a band uniform that selects band b: cdf_f[b] itself selects b + 1,
        # just below it selects b (or 0 below cdf_f[0])
        ub = np.float32(np.nextafter(cdf_f[b], np.float32(0)))
        gcdf = a["probg"][row, b]
        ug = edge_uniforms(gcdf, seed=b, n_random=50)
        nb, g, _, _, _, _ = O.sample_bands(p, tabs, T, 0, np.full_like(ug, ub), ug)
        assert np.all(nb == ref_bisect(cdf_f, ub))
        assert np.array_equal(g, [ref_bisect(a["probg"][row, nb[0]], x) for x in ug])


@pytest.mark.parametrize("grey", [False, True])
def test_wall_search_uses_the_wall_cdf_edge_and_can_take_the_reference_one(grey):
    p, tabs, T = _problem(grey)
    _, _, cdf_f, cdf_s, probq, _ = O.sample_bands(p, tabs, T, 1, [0.5], [0.5])
    u = np.unique(np.concatenate([edge_uniforms(cdf_s), edge_uniforms(cdf_f[:1], n_random=0)]))
    nb, _, _, _, _, _ = O.sample_bands(p, tabs, T, 1, u, np.full_like(u, 0.5))
    assert np.array_equal(nb, [ref_bisect(cdf_s, x) for x in u])
    nb_ref, _, _, _, _, _ = O.sample_bands(p, tabs, T, 1, u, np.full_like(u, 0.5), ref_wall_edge=True)
    assert np.array_equal(nb_ref, [ref_bisect(cdf_s, x, edge0=cdf_f[0]) for x in u])
    # the two rules differ exactly between the two first entries
    lo, hi = sorted((cdf_f[0], cdf_s[0]))
    differ = nb != nb_ref
    assert np.array_equal(differ, (u >= lo) & (u < hi) & (u != 1))
    if not grey:
        ug = edge_uniforms(probq, n_random=50)
        _, g, _, _, _, _ = O.sample_bands(p, tabs, T, 2, np.full_like(ug, 0.5), ug)
        assert np.array_equal(g, [ref_bisect(probq, x) for x in ug])
