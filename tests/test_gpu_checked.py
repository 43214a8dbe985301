"""The bounds-checked build (libradchan_checked.so, RC_CHECKED=1): every
table, field and partial-sum index of the march is checked against its
array on the device.  Small cases covering each path (grey, narrow band
with levels, every wall type, both wall fluxes, a z slab, band-sorted
order, the FP64 build, particle scattering, a batch, the server, the
allocation-free solve) run
in a child process that loads the checked library; none may flag an index
(status bit 3) and each result must equal the oracle bit for bit."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _cases():
    from radchan_b200 import workloads as W
    tabs = W.tables_nb(nB=24, nQ=4, nT=32)
    lv = dict(nB=24, nQ=4, nT=32, levels=[(16, 8, 8), (8, 4, 4)], maxs=[5, 100000])
    out = [("grey", W.channel_params(16, 8, 8, grey=True, photmax=16, nVar=2), None, {}),
           ("nb_levels_walls", W.channel_params(16, 8, 8, photmax=16, nVar=2, calcwalls=1, adiabw=1, adiabe=1, **lv),
            tabs, {}),
           ("black_y_specular_z", W.channel_params(16, 8, 8, photmax=16, nVar=2, bd_y=2, bd_z=3, **lv), tabs, {}),
           ("specular_y_adiabatic_west", W.channel_params(16, 8, 8, photmax=16, nVar=2, bd_y=3, calcwalls=1,
                                                          adiabw=1, **lv), tabs, {}),
           ("sorted", W.channel_params(16, 8, 8, photmax=16, nVar=2, **lv), tabs, {"sort": 1}),
           ("fp64", W.channel_params(16, 8, 8, photmax=8, nVar=2, floatpoint=1, **lv), tabs, {})]
    p = W.channel_params(16, 8, 8, photmax=16, nVar=2, calcwalls=1, adiabw=1, **lv)
    p.p_col = 2
    out.append(("z_slab", p, tabs, {"zstart": 5}))
    out.append(("scattering", W.channel_params(16, 8, 8, photmax=16, nVar=2, bd_y=3, calcwalls=1, adiabw=1,
                                               adiabe=1, **lv), tabs, {"scatter": 1}))
    return out


def child():
    from oracle import oracle as O
    from radchan_b200 import _lib as L
    from radchan_b200 import api
    from radchan_b200 import workloads as W
    assert L.LIB_PATH.endswith("libradchan_checked.so"), L.LIB_PATH
    res = {}
    for name, p, tabs, opt in _cases():
        T = W.channel_field(p, seed=3)
        s = api.Solver(p, tabs)
        if opt.get("sort"):
            s.set_launch(sort_bands=1)
        sc = None
        if opt.get("scatter"):
            sc = api.Scattering.synthetic(nB=24, nQ=4, nA=61, ksca_lo=0.3, ksca_hi=5.0, g_lo=-0.3, g_hi=0.8)
            s.set_scattering(sc)
        z = opt.get("zstart", 1)
        t = s.solve_async(T, zstart=z)
        st = s.info(t).status
        r = s.collect(t)
        o = O.solve(p, tabs, T, zstart=z, rpt=s.get_launch()[0], fp64=bool(p.floatpoint),
                    scatter=sc.arrays() if sc is not None else None)
        res[name] = dict(status=st, equal=bool(np.array_equal(r.q64, o["q64"]) and np.array_equal(r.qw64, o["qw64"])))
        s.close()
    # a batch of two problems and a served request
    cases = _cases()
    b = api.Batch()
    solvers = []
    for name, p, tabs, opt in cases[:2]:
        s = api.Solver(p, tabs)
        solvers.append((s, p, tabs))
        b.add(s, W.channel_field(p, seed=3))
    b.run()
    b.wait()
    eq = True
    for i, (s, p, tabs) in enumerate(solvers):
        o = O.solve(p, tabs, W.channel_field(p, seed=3), rpt=s.get_launch()[0])
        eq = eq and bool(np.array_equal(b.collect(i).q64, o["q64"]))
    b.close()
    res["batch"] = dict(status=0, equal=eq)
    name, p, tabs, _ = cases[1]
    T = W.channel_field(p, seed=3)
    alone = api.Solver(p, tabs).solve(T, want64=False)
    srv = api.Server()
    r = srv.wait(srv.submit(p, T, table_set=srv.add_tables(tabs)))
    srv.close()
    res["server"] = dict(status=0, equal=bool(np.array_equal(r.Q, alone.Q)))
    # the allocation-free entry point reports status bit 3 through its return
    # code (RC_E_RANGE) and message
    import ctypes as C
    import torch
    s = api.Solver(p, tabs)
    dp = lambda t: C.c_void_p(t.data_ptr())
    kl = p.kmax // p.p_col
    q = torch.full((kl, p.jmax, p.imax), float("nan"), dtype=torch.float64, device="cuda")
    v, qw = torch.full_like(q, float("nan")), torch.full((2, kl, p.jmax), float("nan"), dtype=torch.float64,
                                                         device="cuda")
    vw = torch.full_like(qw, float("nan"))
    rc = L.lib().rc_solve_noalloc(s.ctx, dp(torch.from_numpy(T).cuda()), 1, dp(q), dp(v), dp(qw), dp(vw))
    msg = L.last_error(s.ctx) if rc else ""
    o = O.solve(p, tabs, T, rpt=s.get_launch()[0])
    res["noalloc"] = dict(status=8 if "out of bounds" in msg else (0 if rc == 0 else -1), rc=rc, msg=msg,
                          equal=bool(np.array_equal(q.cpu().numpy(), o["q64"]) and
                                     np.array_equal(qw.cpu().numpy(), o["qw64"])))
    s.close()
    print(json.dumps(res))


@pytest.mark.gpu
def test_checked_build_flags_nothing_and_matches_the_oracle():
    from radchan_b200 import build
    build.build(checked=True)   # incremental: relinks only when a source is newer
    env = dict(os.environ, RADCHAN_LIB="checked", PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--child"], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(res) == 11
    for name, v in res.items():
        assert v["status"] >= 0, (name, v)
        assert v["status"] & 8 == 0, (name, v["status"] >> 8)
        assert v["equal"], name


if __name__ == "__main__" and "--child" in sys.argv:
    sys.path.insert(0, ROOT)
    child()
