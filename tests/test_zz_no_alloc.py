"""rc_solve_noalloc: a solve whose scratch is a library-owned static device
array, for callers that cannot allocate device memory while they run.

Its results must equal those of the allocating entry point bit for bit
(same launch knobs, hence the same FP64 summation order) on two calls in a
row, both when this file runs alone in a fresh process and after the other
tests; with one x wall's flux not computed, that wall's rows read 0 as
they do from rc_collect.  A field outside the table range is reported by
the return code (the solve has no ticket to read rc_solve_info from).
This file sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from radchan_b200 import _lib as L
from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev_ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(s, T_dev, q, v, qw, vw, zstart=1):
    return L.lib().rc_solve_noalloc(s.ctx, _dev_ptr(T_dev), zstart, _dev_ptr(q), _dev_ptr(v), _dev_ptr(qw),
                                    _dev_ptr(vw))


@pytest.mark.parametrize("grey,adiabe", [(True, 1), (False, 1), (False, 0)])
def test_noalloc_matches_allocating_solve_twice(grey, adiabe):
    import torch
    tabs = None if grey else W.tables_nb(nB=40, nQ=8, nT=64)
    p = W.channel_params(24, 16, 16, grey=grey, photmax=32, nVar=3, nB=40, levels=[(24, 16, 16), (12, 8, 8)],
                         maxs=[5, 100000], calcwalls=1, adiabw=1, adiabe=adiabe)
    T = W.channel_field(p)
    s = api.Solver(p, tabs)
    ref = s.solve(T)
    T_dev = torch.from_numpy(T).cuda()
    kl = p.kmax // p.p_col
    for call in range(2):
        # outputs start as NaN: every element must be written by the call
        q = torch.full((kl, p.jmax, p.imax), float("nan"), dtype=torch.float64, device="cuda")
        v = torch.full_like(q, float("nan"))
        qw = torch.full((2, kl, p.jmax), float("nan"), dtype=torch.float64, device="cuda")
        vw = torch.full_like(qw, float("nan"))
        L.check(_noalloc(s, T_dev, q, v, qw, vw), s.ctx)
        assert np.array_equal(q.cpu().numpy(), ref.q64)
        assert np.array_equal(v.cpu().numpy(), ref.var64)
        assert np.array_equal(qw.cpu().numpy(), ref.qw64)
        assert np.array_equal(vw.cpu().numpy(), ref.vw64)
    if not adiabe:
        assert not ref.qw64[1].any() and not ref.vw64[1].any()
    s.close()


def test_noalloc_reports_a_field_outside_the_table_range():
    import torch
    tabs = W.tables_nb(nB=40, nQ=8, nT=64)     # tables span 300..2000 K
    p = W.channel_params(24, 16, 16, photmax=16, nVar=2, nB=40)
    T = W.channel_field(p)
    T[5, 6, 7] = 250.0                     # below the first table row
    s = api.Solver(p, tabs)
    t = s.solve_async(T)
    assert s.info(t).status & 1
    ref = s.collect(t)
    T_dev = torch.from_numpy(T).cuda()
    q = torch.full((p.kmax, p.jmax, p.imax), float("nan"), dtype=torch.float64, device="cuda")
    v = torch.full_like(q, float("nan"))
    rc = L.lib().rc_solve_noalloc(s.ctx, _dev_ptr(T_dev), 1, _dev_ptr(q), _dev_ptr(v), None, None)
    assert rc == -6
    assert "table range" in L.last_error(s.ctx)
    assert np.array_equal(q.cpu().numpy(), ref.q64)
    s.close()


def test_noalloc_rejects_problems_beyond_the_scratch_limit():
    import torch
    p = W.channel_params(64, 64, 64, grey=True, photmax=6000, nVar=4)
    s = api.Solver(p)
    s.set_launch(rays_per_thread=2)
    T_dev = torch.from_numpy(W.channel_field(p)).cuda()
    q = torch.zeros((64, 64, 64), dtype=torch.float64, device="cuda")
    v = torch.zeros_like(q)
    rc = L.lib().rc_solve_noalloc(s.ctx, _dev_ptr(T_dev), 1, _dev_ptr(q), _dev_ptr(v), None, None)
    assert rc == -1
    assert "static array" in L.last_error(s.ctx)
    s.close()
