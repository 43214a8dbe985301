"""The benchmark's multi-GPU path runs one independent replica per rank
(replicas only: one solve never spans GPUs) and reports the units of all
ranks over the slowest rank's time.  Exercised here with two gloo ranks on
the CPU: the max-over-ranks reduction and the whole-job aggregation."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    # rank r took (r + 1) seconds for 1000 units
    t = bench.allreduce_max(float(rank + 1), ws)
    v = bench.replica_value(1000.0, float(rank + 1), ws)
    bench.barrier(ws)
    out.put((rank, t, v))
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_whole_job_value():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ws = 2
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == 2.0               # the slowest rank
        assert v == 1000.0 * 2 / 2.0  # all ranks' units over that time
