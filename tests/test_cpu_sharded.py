"""One solve over the ranks of a process group (radchan_b200.sharded), with
two and three gloo ranks on the CPU: rank 0's field is broadcast, each rank
solves its z slab (mc_gpu_noint.cu:97 decomposition), and the gathered
solution on every rank is the whole one.  The per-rank solver is a
deterministic stand-in whose slab result is a function of the field and
the global cell index, so the assembly is checked exactly."""
import datetime
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from radchan_b200 import api
from radchan_b200 import sharded
from radchan_b200 import workloads as W


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _expected(T, k0, k1):
    """The stand-in's answer for cell planes k0..k1 (1-based) of field T."""
    kk = np.arange(k0, k1 + 1)[:, None, None]
    jj = np.arange(1, T.shape[1] - 1)[None, :, None]
    ii = np.arange(1, T.shape[2] - 1)[None, None, :]
    core = T[k0:k1 + 1, 1:-1, 1:-1].astype(np.float64)
    q = 1.5 * core + (ii + 1000 * jj + 1000000 * kk)
    v = 0.25 * core
    qw = np.stack([T[k0:k1 + 1, 1:-1, 0], -T[k0:k1 + 1, 1:-1, -1]]).astype(np.float64)
    return q, v, qw, 0.5 * np.abs(qw)


class FakeSolver:
    def __init__(self, p, tables, device):
        self.p = p
        self.kloc = p.kmax // p.p_col

    def solve_async(self, T, zstart=1):
        self.T = np.array(T)
        self.z = zstart
        return 1

    def collect(self, ticket, want64=True):
        q, v, qw, vw = _expected(self.T, self.z, self.z + self.kloc - 1)
        return api.Result(None, None, q, v, qw, vw)

    def close(self):
        pass


def _worker(rank, ws, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    p = W.channel_params(12, 8, 6 * ws, calcwalls=1, adiabw=1, adiabe=1)
    T = W.channel_field(p, seed=5) if rank == 0 else None
    s = sharded.ShardedSolver(p, None, solver_factory=FakeSolver)
    r = s.solve(T)
    s.close()
    out.put((rank, s.zstart, s.kloc, r.q64, r.var64, r.qw64, r.vw64))
    dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_gloo_ranks_gather_the_whole_solution(ws):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=120) for _ in range(ws)), key=lambda x: x[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p = W.channel_params(12, 8, 6 * ws)
    T = W.channel_field(p, seed=5)
    want = _expected(T, 1, p.kmax)
    for rank, zstart, kloc, *got in res:
        assert (zstart, kloc) == (rank * 6 + 1, 6)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


def test_slab_arithmetic():
    assert sharded.slab(64, 1, 0) == (64, 1)
    assert sharded.slab(64, 4, 3) == (16, 49)
    with pytest.raises(ValueError):
        sharded.slab(64, 3, 0)
    with pytest.raises(ValueError):
        sharded.slab(64, 4, 4)


def test_fortran_layout_of_a_gathered_result():
    p = W.channel_params(5, 4, 3, calcwalls=1, adiabw=1, adiabe=0)
    rng = np.random.default_rng(0)
    r = sharded.ShardedResult(rng.standard_normal((3, 4, 5)), rng.random((3, 4, 5)),
                              rng.standard_normal((2, 3, 4)), rng.random((2, 3, 4)))
    Q, S = r.fortran(p)
    assert Q.shape == (5, 6, 7) and Q.dtype == np.float32
    np.testing.assert_array_equal(Q[1:-1, 1:-1, 1:-1], r.q64.astype(np.float32))
    np.testing.assert_array_equal(S[1:-1, 1:-1, 1:-1], np.sqrt(r.var64).astype(np.float32))
    np.testing.assert_array_equal(Q[1:-1, 1:-1, 0], r.qw64[0].astype(np.float32))
    assert np.all(Q[1:-1, 1:-1, -1] == 0)   # east flux not computed
    assert np.all(Q[0] == 0) and np.all(Q[:, 0] == 0)


# ---- the same decomposition behind the C ABI (rc_slab_*, NCCL loaded by the
#      library): what runs without a GPU

def test_native_slab_range_matches_the_python_decomposition():
    for kmax in (1, 6, 64, 2304):
        for ws in (1, 2, 3, 4, 8):
            for rank in range(ws):
                if kmax % ws:
                    with pytest.raises(api.L.RadChanError):
                        api.slab_range(kmax, ws, rank)
                else:
                    assert api.slab_range(kmax, ws, rank) == sharded.slab(kmax, ws, rank)
    for bad in ((64, 4, 4), (64, 0, 0), (64, 2, -1), (0, 1, 0)):
        with pytest.raises(api.L.RadChanError) as e:
            api.slab_range(*bad)
        assert e.value.code == -1


def test_native_slab_group_ids_and_argument_checks():
    import ctypes as C
    a, b = api.slab_unique_id(), api.slab_unique_id()
    assert len(a) == 128 and a != b
    lib = api.L.lib()
    comm = C.c_void_p()
    assert lib.rc_slab_comm_create(0, 0, 0, a, 1.0, C.byref(comm)) == -1
    assert lib.rc_slab_comm_create(0, 2, 2, a, 1.0, C.byref(comm)) == -1
    assert lib.rc_slab_comm_create(0, 1, 0, None, 1.0, C.byref(comm)) == -1
    assert not comm.value
    assert lib.rc_slab_solve(None, None, None, None, None, None, None) == -1
    assert lib.rc_slab_comm_destroy(None) == 0


def test_native_slab_reports_a_missing_nccl():
    """Without an NCCL to load, the group calls fail with RC_E_NOTFOUND and
    say which file was tried (the rest of the library works without it)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("from radchan_b200 import api\n"
            "try:\n"
            "    api.slab_unique_id()\n"
            "except api.L.RadChanError as e:\n"
            "    assert e.code == -8 and 'cannot load NCCL' in str(e) and 'no_such_nccl' in str(e), str(e)\n"
            "    print('refused')\n"
            "print(api.slab_range(8, 2, 1))\n")
    env = dict(os.environ, RC_NCCL_LIBRARY="/nonexistent/no_such_nccl.so")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["refused", "(4,", "5)"]
