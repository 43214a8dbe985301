"""One solve over several GPUs by z slabs: the slabs of a p_col
decomposition (mc_gpu_noint.cu:97) reproduce the one-GPU solve exactly, so
gathering them is the whole solution; and the ShardedSolver's device path
(NCCL broadcast, device solve, device collect, all-gather) equals the plain
solve on a one-rank NCCL group."""
import datetime
import socket

import numpy as np
import pytest

from radchan_b200 import api
from radchan_b200 import sharded
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _problem():
    tabs = W.tables_nb(nB=40, nQ=4, nT=32)
    p = W.channel_params(32, 16, 24, photmax=32, nVar=4, nB=40, nQ=4, nT=32,
                         levels=[(32, 16, 24), (16, 8, 12)], maxs=[5, 100000], calcwalls=1, adiabw=1, adiabe=1)
    return p, tabs, W.channel_field(p, seed=8)


@pytest.mark.parametrize("n", [2, 3, 4])
def test_slabs_concatenate_to_the_one_gpu_solve(n):
    p, tabs, T = _problem()
    full = api.Solver(p, tabs)
    r = full.solve(T)
    full.close()
    q = api.copy_params(p)
    q.p_col = n
    parts = []
    for rank in range(n):
        kloc, z = sharded.slab(p.kmax, n, rank)
        s = api.Solver(q, tabs)
        parts.append(s.solve(T, zstart=z))
        s.close()
    np.testing.assert_array_equal(np.concatenate([x.q64 for x in parts]), r.q64)
    np.testing.assert_array_equal(np.concatenate([x.var64 for x in parts]), r.var64)
    np.testing.assert_array_equal(np.concatenate([x.qw64 for x in parts], axis=1), r.qw64)
    np.testing.assert_array_equal(np.concatenate([x.vw64 for x in parts], axis=1), r.vw64)


def test_sharded_solver_device_path_on_a_one_rank_nccl_group():
    import torch
    import torch.distributed as dist
    p, tabs, T = _problem()
    ref = api.Solver(p, tabs).solve(T)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sh = sharded.ShardedSolver(p, tabs)
        assert sh.nccl and (sh.kloc, sh.zstart) == (p.kmax, 1)
        r = sh.solve(T)
        sh.close()
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(r.q64, ref.q64)
    np.testing.assert_array_equal(r.var64, ref.var64)
    np.testing.assert_array_equal(r.qw64, ref.qw64)
    np.testing.assert_array_equal(r.vw64, ref.vw64)
    Q, S = r.fortran(p)
    np.testing.assert_array_equal(Q[1:-1, 1:-1, :], ref.Q[1:-1, 1:-1, :])
    np.testing.assert_array_equal(S[1:-1, 1:-1, :], ref.sigma[1:-1, 1:-1, :])
