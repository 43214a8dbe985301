"""Benchmark of the OERM Monte Carlo radiative source on B200.

Default workload: narrow-band correlated-k 64^3 channel (100 bands x 8 g,
64 temperatures, 3 multigrid levels 64/32/16 with maxs 5/5/1e5,
photmax 256, nVar 4, band-sorted order, adiabatic west wall with wall-flux
kernel), seeded synthetic field and tables.  One step = one full solve.

  value  photon bundles/s with the field already in HBM (device time of the
         solve: copy-in, set-up, march, tally), max over ranks, summed over
         ranks (replicas: one independent solve per GPU);
  e2e    the same through the public API with host buffers: rc_solve_async
         from a host array + rc_collect into host arrays, wall clock;
  roofline  march kernel: ray-cell steps x 32 B (one sector per temperature
         gather) / march time vs the measured HBM copy bandwidth.

--impl reference times the CPU restatement of the reference's ray loop
(the reference has no CPU implementation of this path) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BUNDLE_METRIC = "bundles/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(name, photmax=0):
    from radchan_b200 import workloads as W
    if name == "nb64":
        p = W.config_nb_64(photmax=photmax or 256)
        tabs = W.tables_nb()
        desc = dict(workload="narrow-band 100x8 OERM, 64^3 channel, 3 levels 64/32/16 maxs 5/5/1e5, photmax %d, "
                             "nVar 4, srt 1, calcwalls (adiabatic west wall)" % p.photmax,
                    grid=[64, 64, 64], bands=100, gpoints=8, temps=64, photmax=p.photmax, nVar=4, levels=3)
    elif name == "grey32":
        p = W.config_grey_32(photmax=photmax or 64)
        tabs = None
        desc = dict(workload="grey OERM kappa=1, 32^3 channel, photmax 64, nVar 4", grid=[32, 32, 32], photmax=64,
                    nVar=4, levels=1)
    else:
        raise SystemExit("unknown workload " + name)
    T = W.channel_field(p)
    return p, tabs, T, desc


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.path = os.path.join("/tmp", "rc_clocks_%d_%d.csv" % (os.getpid(), dev))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(p, tabs, T, seconds=12.0, nthreads=0):
    """Oracle (CPU restatement) on a bounded sample of the workload's cells."""
    from oracle import oracle as O
    ncells = p.imax * p.jmax * (p.kmax // p.p_col)
    n = 64
    t0 = time.perf_counter()
    r = O.solve(p, tabs, T, rpt=8, cell_begin=0, cell_end=n, walls=False, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n2 = int(min(ncells, max(n, n * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    r = O.solve(p, tabs, T, rpt=8, cell_begin=0, cell_end=n2, walls=False, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return dict(bundles=r["bundles"], steps=r["steps"], seconds=dt, cells=n2)


def run_reference(args, ws, rank):
    if rank != 0:
        return
    p, tabs, T, desc = workload(args.workload, args.photmax)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(p, tabs, T, seconds=1.0)
    tot_b, tot_s, tot_t = 0.0, 0.0, 0.0
    cells = 0
    for _ in range(args.steps):
        r = cpu_sample(p, tabs, T, seconds=args.ref_seconds)
        tot_b += r["bundles"]
        tot_s += r["steps"]
        tot_t += r["seconds"]
        cells = r["cells"]
    v = tot_b / tot_t
    sample = "%d of %d fluid cells x nVar %d x photmax %d per step (walls excluded), %d steps" % (
        cells, p.imax * p.jmax * p.kmax, p.nVar, p.photmax, args.steps)
    line = {"impl": "reference", "metric": BUNDLE_METRIC, "value": v, "unit": "bundles/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(desc, parallelism="replicas"),
            "steps_per_s": tot_s / tot_t,
            "cpu_baseline": {"value": v, "unit": "bundles/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "bundles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch

    from radchan_b200 import api
    p, tabs, T, desc = workload(args.workload, args.photmax)
    dev = local
    torch.cuda.set_device(dev)
    s = api.Solver(p, tabs, device=dev)
    if args.rays_per_thread or args.block or args.occupancy:
        s.set_launch(rays_per_thread=args.rays_per_thread, block_threads=args.block, occupancy=args.occupancy)
    T_dev = torch.from_numpy(T).to(f"cuda:{dev}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    # k_init_scalars, k_tmax, k_setup1, k_setup2, k_levels, k_patch_desc,
    # k_march, k_tally (+ k_grey_ib, k_build_ki for a grey gas)
    kernels_per_solve = 8 + (2 if p.grey else 0)
    # warm-up
    for _ in range(args.warmup):
        t = s.solve_device_async(T_dev.data_ptr())
        s.wait_device(t)
        s.release(t)
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    ms_solve, ms_march, bundles, steps = [], [], 0.0, 0.0
    rel_std = None
    t_wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the solve's events)
        torch.cuda.synchronize()
        t = s.solve_device_async(T_dev.data_ptr())
        info = s.info(t)
        ms_solve.append(info.ms_solve)
        ms_march.append(info.ms_device)
        bundles += info.bundles
        steps += info.steps
        if k == args.steps - 1:
            r = s.collect(t)
            i = np.unravel_index(np.argmax(np.abs(r.q64)), r.q64.shape)
            rel_std = float(np.sqrt(r.var64[i]) / abs(r.q64[i]))
        else:
            s.release(t)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    barrier(ws)
    t_dev = sum(ms_solve) / 1000.0
    t_max = allreduce_max(t_dev, ws)
    value = bundles * ws / t_max
    # e2e through the public API with host buffers
    Qh = np.zeros(api.result_shape(p), np.float32)
    Sh = np.zeros(api.result_shape(p), np.float32)
    for _ in range(max(1, args.warmup)):
        s.collect_into(s.solve_async(T), Qh, Sh)
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.collect_into(s.solve_async(T), Qh, Sh)
    t_e2e = allreduce_max(time.perf_counter() - t0, ws)
    kl = p.kmax // p.p_col
    d2h = (2 * p.imax * p.jmax * kl + 4 * p.jmax * kl) * 4
    e2e = {"value": bundles * ws / t_e2e, "unit": "bundles/s", "h2d_bytes_per_step": int(T.nbytes),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": 1000 * t_e2e / args.steps}
    peak, peak_kind = peaks()
    march_s = sum(ms_march) / 1000.0
    achieved = steps * 32.0 / march_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": args.traffic, "kernel": "k_march", "peak_source": peak_kind,
            "algorithmic_bytes_per_step": 32, "steps_per_launch": steps / args.steps}
    line = {"metric": BUNDLE_METRIC, "value": value, "unit": "bundles/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(desc, parallelism="replicas" if ws > 1 else "single", l2="flushed between steps"),
            "steps_per_s": steps * ws / t_max, "solves_per_s": args.steps * ws / t_max,
            "rel_std_maxq": rel_std, "march_ms": 1000 * march_s / args.steps,
            "roofline": roof, "e2e": e2e, "gpu_launches": kernels_per_solve * args.steps,
            "clocks": clk, "wall_s": wall}
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_sample(p, tabs, T, seconds=args.ref_seconds)
        line["cpu_baseline"] = {"value": cb["bundles"] / cb["seconds"], "unit": "bundles/s",
                                "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": "%d fluid cells x nVar %d x photmax %d (walls excluded), %.1f s" % (
                                    cb["cells"], p.nVar, p.photmax, cb["seconds"])}
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="nb64")
    ap.add_argument("--rays-per-thread", dest="rays_per_thread", type=int, default=0)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--occupancy", type=int, default=0)
    ap.add_argument("--ref-seconds", dest="ref_seconds", type=float, default=12.0)
    ap.add_argument("--traffic", type=float, default=None)
    ap.add_argument("--photmax", type=int, default=0, help="override bundles per cell (profiling runs)")
    ap.add_argument("--no-cpu-baseline", dest="no_cpu_baseline", action="store_true")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
