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


def test_native_slab_group_of_one_equals_the_plain_solve():
    """rc_slab_solve on a one-rank group (NCCL inside the library): device
    arrays, host arrays and no wall outputs all give the plain solve bit for
    bit; a context of another decomposition and a non-finite field are
    reported, and the group stays usable after both."""
    import torch
    p, tabs, T = _problem()
    s = api.Solver(p, tabs)
    ref = s.solve(T)
    comm = api.SlabComm(0, 1, 0, api.slab_unique_id(), timeout_s=60)
    try:
        Td = torch.from_numpy(T).cuda()
        f64 = dict(dtype=torch.float64, device="cuda")
        q, v = torch.empty((p.kmax, p.jmax, p.imax), **f64), torch.empty((p.kmax, p.jmax, p.imax), **f64)
        qw, vw = torch.empty((2, p.kmax, p.jmax), **f64), torch.empty((2, p.kmax, p.jmax), **f64)
        comm.solve(s, Td.data_ptr(), q.data_ptr(), v.data_ptr(), qw.data_ptr(), vw.data_ptr())
        torch.cuda.synchronize()
        for got, want in ((q, ref.q64), (v, ref.var64), (qw, ref.qw64), (vw, ref.vw64)):
            np.testing.assert_array_equal(got.cpu().numpy(), want)
        hq, hv, hqw, hvw = comm.solve_arrays(s, T)
        for got, want in ((hq, ref.q64), (hv, ref.var64), (hqw, ref.qw64), (hvw, ref.vw64)):
            np.testing.assert_array_equal(got, want)
        q.zero_()
        comm.solve(s, Td.data_ptr(), q.data_ptr(), v.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(q.cpu().numpy(), ref.q64)

        other = api.copy_params(p)
        other.p_col = 2
        s2 = api.Solver(other, tabs)
        with pytest.raises(api.L.RadChanError) as e:
            comm.solve_arrays(s2, T)
        assert e.value.code == -1 and "p_col" in str(e.value)
        s2.close()
        Tbad = T.copy()
        Tbad[3, 3, 3] = np.nan
        with pytest.raises(api.L.RadChanError) as e:
            comm.solve_arrays(s, Tbad)
        assert e.value.code == -6
        hq, *_ = comm.solve_arrays(s, T)
        np.testing.assert_array_equal(hq, ref.q64)
    finally:
        comm.close()
        s.close()


def test_native_slab_group_whose_peer_never_joins_times_out():
    """Rank 0 of a two-rank group whose rank 1 never starts: joining ends
    with RC_E_TIMEOUT after the communicator's timeout and the group is
    abandoned (host side only: no collective is ever launched).  Run in a
    child process with NVLS off."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import time\n"
            "from radchan_b200 import api\n"
            "t0 = time.time()\n"
            "try:\n"
            "    api.SlabComm(0, 2, 0, api.slab_unique_id(), timeout_s=3.0)\n"
            "except api.L.RadChanError as e:\n"
            "    assert e.code == -10, str(e)\n"
            "    print('timeout', round(time.time() - t0))\n")
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    # (NCCL may print its version banner first)
    words = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("timeout ")]
    assert len(words) == 1 and 3 <= int(words[0][1]) <= 60, r.stdout
