"""Benchmark of the OERM Monte Carlo radiative source on B200.

Default workload: narrow-band correlated-k 64^3 channel (100 bands x 8 g,
64 temperatures, 3 multigrid levels 64/32/16 with maxs 5/5/1e5,
photmax 256, nVar 4, srt 1 in the parameter set, adiabatic west wall with
wall-flux kernel), seeded synthetic field and tables.  One step = one full
solve.

  value  photon bundles/s with the field already in HBM (device time of the
         solve: copy-in, set-up, march, tally), max over ranks, summed over
         ranks (replicas: one independent solve per GPU);
  e2e    the same through the public API with host buffers: rc_solve_async
         from a host array + rc_collect into host arrays, wall clock, with
         the next solve issued before the previous one is collected (the
         context's two slots);
  roofline  march kernel: ray-cell steps x 32 B (one sector per temperature
         gather) / march time vs the measured HBM copy bandwidth.

Legs on one GPU (skipped with --no-legs):
  at_1pct  the same solve with photmax raised until the relative std of
         max|Q| is 1%: solves/s and bundles/s at that tolerance;
  batched  64 uneven problems (grids 16..96 per axis, half grey, half
         narrow-band 20-100 bands, photmax 32/128/512): plain one solve per
         launch vs one persistent launch from a CUDA graph vs the
         continuous-batching server, solves/s by wall clock;
  batched_small  the same with edges 16..32 and photmax 32/128;
  dns_source  the DNS coupling kernel (Q, sigma -> Qnew, Varnew, Knew,
         Gnew) on the 192x128x128 channel: device time per launch, HBM
         roofline, host entry point time, CPU restatement time;
  batched_at_1pct, batched_small_at_1pct  the two mixes at equal 1%
         relative std of max|Q| (photmax per problem from a pilot);
  scattering  the benchmark solve with particle scattering added, next to
         the same solve without particles;
  serve  the open-loop serving stream below, capped in wall time.

--serve runs the open-loop serving benchmark instead (Poisson arrivals at
--load x measured capacity, tolerance-driven photmax, p50/p99 latency);
--precision runs the FP32-march vs FP64-build study at 192x128x128;
--dns-leg and --scatter-leg run one leg alone (profiling runs);
--workload c4 runs the march on the precision study's 192x128x128 channel.

--impl reference times the CPU restatement of the reference's ray loop
(the reference has no CPU implementation of this path) on all host cores,
on inputs the oracle builds itself (the product library is never loaded),
and then the reference's own CUDA build on the same GPU (ref_cuda: each
solve in a child process, since get_results_ resets the device).
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

BUNDLE_METRIC = "bundles/s & solves/s at 1% MC std, batched/served vs plain; serve p50/p99"

# DRAM bytes (read + write) of one k_march launch, from the ncu capture
# summarised in profiles/k_march_nb64_photmax64_full.txt
# (dram__bytes_read.sum + dram__bytes_write.sum).  The march's working set
# (temperature pyramid and tables, ~1.5 MB) is L2-resident, so the traffic
# does not grow with photmax.
K_MARCH_TRAFFIC = {"nb64": 1597184 + 0}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_desc(name, p):
    """The config dict of a workload, from its parameter set (either the
    product's or the oracle's rc_params mirror)."""
    if name == "nb64":
        return dict(workload="narrow-band 100x8 OERM, 64^3 channel, 3 levels 64/32/16 maxs 5/5/1e5, photmax %d, "
                             "nVar 4, srt 1, calcwalls (adiabatic west wall)" % p.photmax,
                    grid=[64, 64, 64], bands=100, gpoints=8, temps=64, photmax=p.photmax, nVar=4, levels=3)
    if name == "grey32":
        return dict(workload="grey OERM kappa=1, 32^3 channel, photmax %d, nVar 4" % p.photmax, grid=[32, 32, 32],
                    photmax=p.photmax, nVar=4, levels=1)
    if name == "c4":
        return dict(workload="narrow-band 100x8 OERM, optically thick, 192x128x128 channel, specular y, "
                             "photmax %d, nVar %d" % (p.photmax, p.nVar), grid=[192, 128, 128], bands=100, gpoints=8,
                    temps=64, photmax=p.photmax, nVar=p.nVar, levels=p.grid_num)
    raise SystemExit("unknown workload " + name)


def bench_config(desc, ws):
    """The same config dict in both arms."""
    return dict(desc, parallelism="replicas" if ws > 1 else "single", l2="flushed between steps")


def workload(name, photmax=0):
    """Seeded inputs built by the product package (this solver's arm)."""
    from radchan_b200 import workloads as W
    if name == "nb64":
        p = W.config_nb_64(photmax=photmax or 256)
        tabs = W.tables_nb()
    elif name == "grey32":
        p = W.config_grey_32(photmax=photmax or 64)
        tabs = None
    elif name == "c4":
        # the precision study's channel (192x128x128, optically thick tables,
        # emissivity 0.8, specular y walls): profiling runs of the march on a
        # 3.1 M-cell pyramid
        p = W.config_precision(photmax=photmax or 1024)
        tabs = W.tables_nb(logk_lo=-1.0, logk_hi=2.0)
    else:
        raise SystemExit("unknown workload " + name)
    return p, tabs, W.channel_field(p), workload_desc(name, p)


def workload_oracle(name, photmax=0):
    """The same inputs built by the oracle alone (the reference arm never
    loads the product library); tests/test_cpu_oracle_workload.py checks
    they are identical byte for byte."""
    from oracle import workload as OW
    if name == "nb64":
        p = OW.params_nb64(photmax=photmax or 256)
        tabs = OW.tables_nb()
    elif name == "grey32":
        p = OW.channel_params(32, 32, 32, grey=True, photmax=photmax or 64)
        tabs = None
    else:
        raise SystemExit("unknown workload " + name)
    return p, tabs, OW.channel_field(p), workload_desc(name, p)


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
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
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
    """Max of a per-rank timing over all ranks (the job is as slow as its
    slowest replica); on the device for NCCL, on the host for gloo."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, seconds, ws):
    """Whole-job throughput of ws independent replicas: the units all ranks
    processed over the slowest rank's time (max over ranks)."""
    return units_per_rank * ws / allreduce_max(seconds, ws)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample(p, tabs, T, seconds=12.0, nthreads=0):
    """Oracle (CPU restatement) on a bounded sample of the workload's cells."""
    from oracle import oracle as O
    ncells = p.imax * p.jmax * (p.kmax // p.p_col)
    n = 64
    for _ in range(5):
        t0 = time.perf_counter()
        r = O.solve(p, tabs, T, rpt=8, cell_begin=0, cell_end=n, walls=False, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if dt >= 0.5 * seconds or n >= ncells:
            break
        n = int(min(ncells, max(2 * n, n * seconds / max(dt, 1e-3))))
    return dict(bundles=r["bundles"], steps=r["steps"], seconds=dt, cells=n)


def ref_cuda_child(lib_path, out_path, photmax):
    """One solve of the reference's own CUDA build (oracle/_ref, built by
    oracle/ref_build.py) in this process: tables written in its file formats
    to a scratch directory (readT reads ./properties on every call), then
    mc_gpu_ + get_results_ timed by oracle/ref_driver.cu."""
    import ctypes as C
    import tempfile

    from oracle import workload as OW
    p, tabs, T, _ = workload_oracle("nb64", photmax)
    wd = tempfile.mkdtemp(prefix="rc_refcuda_")
    OW.write_reference_dir(tabs, os.path.join(wd, "properties"))
    os.chdir(wd)
    lib = C.CDLL(lib_path)
    fp = C.POINTER(C.c_float)
    lib.ref_solve_timed.restype = C.c_int
    lib.ref_solve_timed.argtypes = [fp, C.c_int, fp, fp, C.POINTER(C.c_double)]
    shape = (p.kmax + 2, p.jmax + 2, p.imax + 2)
    Q = np.zeros(shape, np.float32)
    S = np.zeros(shape, np.float32)
    ms = (C.c_double * 4)()
    Tc = np.ascontiguousarray(T)
    rc = lib.ref_solve_timed(Tc.ctypes.data_as(fp), 1, Q.ctypes.data_as(fp), S.ctypes.data_as(fp), ms)
    with open(out_path, "w") as f:
        json.dump({"rc": rc, "ms": list(ms), "finite": bool(np.isfinite(Q).all())}, f)


def leg_ref_cuda(photmax, runs=3):
    """The reference's own CUDA build of the workload (srt 1 as configured)
    on this GPU: each solve in a child process of its own, because
    get_results_ resets the device.  Reported: wall time of mc_gpu_ +
    get_results_ and its parts (mc_gpu_ itself: table files, uploads,
    launches; the kernels still running after it returns; get_results_),
    and bundles/s on the wall clock and on the kernel time."""
    import tempfile
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_nb64.so")
    if not os.path.exists(lib):
        return {"unavailable": "oracle/_ref/libref_nb64.so not built (the reference sources were absent at build)"}
    out = []
    for r in range(runs):
        path = os.path.join(tempfile.mkdtemp(prefix="rc_refcuda_"), "r.json")
        cp = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-cuda-child", lib, path,
                             str(photmax)], capture_output=True, text=True, timeout=600)
        if cp.returncode != 0 or not os.path.exists(path):
            return {"unavailable": "reference CUDA build failed: " + (cp.stderr or cp.stdout)[-300:]}
        out.append(json.load(open(path)))
    ms = np.array([o["ms"] for o in out])
    med = np.median(ms, axis=0)
    bundles = 64 * 64 * 64 * 4 * photmax + 64 * 64 * 4 * photmax   # fluid cells + west-wall cells
    return {"build": "oracle/_ref/libref_nb64.so (reference sources, srt 1 as configured, sm_100a)",
            "runs": runs, "rc": [o["rc"] for o in out], "finite": all(o["finite"] for o in out),
            "ms_wall": float(med[0]), "ms_mc_gpu": float(med[1]), "ms_kernels_after_return": float(med[2]),
            "ms_get_results": float(med[3]), "ms_wall_runs": [float(x) for x in ms[:, 0]],
            "bundles_per_solve": bundles, "bundles_per_s_wall": bundles / (med[0] / 1000.0),
            "bundles_per_s_kernels": bundles / (med[2] / 1000.0),
            "note": "kernels_after_return is the time from mc_gpu_'s return (kernels launched) to device idle"}


def run_reference(args, ws, rank):
    """The reference arm: the CPU restatement of the reference's ray loop
    (the reference has no CPU implementation of this path) on all host cores,
    on inputs the oracle builds itself; then the reference's own CUDA build
    on this GPU (ref_cuda), outside the timed region."""
    if rank != 0:
        return
    p, tabs, T, desc = workload_oracle(args.workload, args.photmax)
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
            "config": bench_config(desc, ws),
            "steps_per_s": tot_s / tot_t,
            "cpu_baseline": {"value": v, "unit": "bundles/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "bundles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "nb64" and not args.no_legs:
        line["ref_cuda"] = leg_ref_cuda(p.photmax)
    print(json.dumps(line), flush=True)


def gather_ceilings(p, achieved_gbs, dev):
    """The march's gathers stay in L2 (the temperature pyramid of every level
    as uint16 coordinates plus the interleaved k / I_b table rows), so next
    to the HBM convention its achieved 32 B/step rate is stated against the
    random-sector gather throughput this GPU delivers over an array of that
    size (rc_probe_gather): L2 only, and through L1 as the march reads."""
    from radchan_b200 import api
    cells = sum(p.maxi[l] * p.maxj[l] * p.maxk[l] for l in range(p.grid_num))
    nB, nQ, nT = (p.grey_nB, 1, p.grey_nT) if p.grey else (p.nB, p.nQ, p.nT)
    ws = 2 * cells + 16 * nB * nQ * nT
    _, l2, _ = api.probe_gather(ws, mode=0, device=dev)
    _, l1l2, _ = api.probe_gather(ws, mode=1, device=dev)
    return {"working_set_bytes": ws, "l2_gather_gbs": l2, "frac_l2": achieved_gbs / l2,
            "l1l2_gather_gbs": l1l2, "frac_l1l2": achieved_gbs / l1l2,
            "gather_probe": "rc_probe_gather: 4 B from a random 32 B sector per lane, 8 in flight, full occupancy; "
                            "GB/s = sectors/s x 32"}


def leg_at_tolerance(p, tabs, T, rel0, dev, flush, tol=0.01, steps=2):
    """The same solve with photmax raised until the relative standard
    deviation of max|Q| is `tol` (it falls as photmax^-1/2): device time per
    solve, solves/s and bundles/s at that tolerance."""
    import math

    import torch

    from radchan_b200 import api
    q = api.copy_params(p)
    q.photmax = int(math.ceil(p.photmax * (rel0 / tol) ** 2))
    s = api.Solver(q, tabs, device=dev)
    T_dev = torch.from_numpy(T).to(f"cuda:{dev}")
    t = s.solve_device_async(T_dev.data_ptr())
    s.wait_device(t)
    s.release(t)
    ms, bundles, rel = [], 0.0, None
    for k in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t = s.solve_device_async(T_dev.data_ptr())
        info = s.info(t)
        ms.append(info.ms_solve)
        bundles += info.bundles
        if k == steps - 1:
            r = s.collect(t)
            rel = api.rel_std_maxq(r.q64, np.sqrt(r.var64))
        else:
            s.release(t)
    s.close()
    sec = sum(ms) / 1000.0
    return {"tolerance": tol, "photmax": q.photmax, "rel_std_maxq": rel, "ms_per_solve": 1000 * sec / steps,
            "solves_per_s": steps / sec, "bundles_per_s": bundles / sec, "steps": steps}


def leg_scattering(p, tabs, T, dev, flush, steps=3):
    """The benchmark solve with particle scattering added (synthetic
    Henyey-Greenstein tables: scattering coefficient log-uniform on
    [0.1, 1] per band, asymmetry g uniform on [0, 0.8], 181 angles): device
    time, bundles/s, ray-cell steps/s (scattering events count as steps)
    next to the same solve without particles."""
    import torch

    from radchan_b200 import api
    s = api.Solver(p, tabs, device=dev)
    T_dev = torch.from_numpy(T).to(f"cuda:{dev}")

    def timed():
        t = s.solve_device_async(T_dev.data_ptr())
        s.wait_device(t)
        s.release(t)
        ms, bundles, nsteps = [], 0.0, 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t = s.solve_device_async(T_dev.data_ptr())
            info = s.info(t)
            ms.append(info.ms_solve)
            bundles += info.bundles
            nsteps += info.steps
            s.release(t)
        sec = sum(ms) / 1000.0
        return {"ms_per_solve": 1000 * sec / steps, "bundles_per_s": bundles / sec, "steps_per_s": nsteps / sec,
                "steps_per_bundle": nsteps / bundles}

    plain = timed()
    sc = api.Scattering.synthetic(nB=p.nB, nQ=p.nQ, nA=181, ksca_lo=0.1, ksca_hi=1.0, g_lo=0.0, g_hi=0.8, seed=3)
    s.set_scattering(sc)
    scat = timed()
    s.close()
    return {"particles": "ksca log-uniform [0.1, 1] 1/m per band, Henyey-Greenstein g ~ U[0, 0.8], 181 angles",
            "with_scattering": scat, "without": plain}


def leg_dns_source(dev, flush, reps=20, cpu=True):
    """The DNS coupling kernel (k_dns_source: GET_RESULTS + fix_rad +
    fix_kappa + the Gnew loop of src/dns/channel.f:249-266) on the
    192x128x128 channel (the largest grid of the workload family), full
    j pencil: device time per launch on the launching stream with L2
    flushed before each launch, HBM roofline at 48 algorithmic bytes per
    output cell (float Q and sigma 8, double T1 8, four double outputs 32);
    the host entry point (T1 in, four arrays out over PCIe) by wall clock;
    the CPU restatement on the same arrays."""
    import torch

    from radchan_b200 import api
    from radchan_b200 import workloads as W
    p = W.config_precision(photmax=1, nVar=2)
    tabs = W.tables_nb()
    a = tabs.arrays()
    Tin = 955.0
    cpl = api.DnsCoupling(Tin=Tin, Height=0.5, underrelax=1.0, Tnb=a["Tnb"].astype(np.float64),
                          kP=a["kP"].astype(np.float64) * 0.5)
    T1 = W.channel_field(p).astype(np.float64) / Tin
    T = api.field_from_dns(T1, Tin)
    s = api.Solver(p, tabs, device=dev)
    tshape, oshape = cpl.pencil_shapes(p)
    cuda = torch.device("cuda:%d" % dev)
    T1d = torch.from_numpy(np.ascontiguousarray(T1)).to(cuda)
    outs = [torch.empty(oshape, dtype=torch.float64, device=cuda) for _ in range(4)]
    cnt = torch.zeros(1, dtype=torch.int64, device=cuda)
    # a stream of its own: handle 0 (torch's legacy default stream) would
    # select the solve's stream in rc_dns_source_device
    stream = torch.cuda.Stream(device=cuda)
    torch.cuda.synchronize(cuda)
    t = s.solve_async(T)
    s.wait_device(t)
    ptrs = [o.data_ptr() for o in outs]
    with torch.cuda.stream(stream):
        for _ in range(3):
            s.dns_source_device(t, cpl, T1d.data_ptr(), *ptrs, cnt.data_ptr(), stream=stream.cuda_stream)
        ms = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.dns_source_device(t, cpl, T1d.data_ptr(), *ptrs, cnt.data_ptr(), stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(cuda)
    r = s.collect(t, want64=False)
    n_out = int(np.prod(oshape))
    sec = sum(ms) / 1000.0 / reps
    peak, peak_kind = peaks()
    achieved = 48.0 * n_out / sec / 1e9
    # host entry point: pencil in, four arrays out, per call after the solve
    host_ms = []
    for _ in range(3):
        t = s.solve_async(T)
        s.wait_device(t)
        t0 = time.perf_counter()
        s.dns_source(t, cpl, T1)
        host_ms.append(1000 * (time.perf_counter() - t0))
    s.close()
    out = {"kernel": "k_dns_source", "grid": [p.imax, p.jmax, p.kmax], "cells": n_out, "launches": reps,
           "ms_per_launch": 1000 * sec,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "algorithmic_bytes_per_cell": 48},
           "host_entry_ms": min(host_ms), "host_entry_bytes": int(T1.nbytes + 32 * n_out),
           "l2": "flushed before each launch"}
    if cpu:
        from oracle import dns as OD
        t0 = time.perf_counter()
        OD.dns_source(r.Q, r.sigma, T1, Tin, cpl.Height, cpl.underrelax, cpl.stefan, cpl.Tnb, cpl.kP, 1, p.jmax)
        out["cpu_baseline"] = {"ms": 1000 * (time.perf_counter() - t0), "cores": 1, "kind": "port",
                               "sample": "the whole pencil, numpy restatement of fixvar.f/channel.f"}
    return out


def batch_setup(dev, n=64, edges=(16, 24, 32, 48, 64, 96), photmaxes=(32, 128, 512)):
    """The uneven-problem mix: 64 problems, grid edges from
    {16,24,32,48,64,96} per axis, half grey and half narrow-band (20-100
    bands x 8 g), photmax from {32,128,512}; seeded fields and tables."""
    from radchan_b200 import api
    from radchan_b200 import workloads as W
    probs = W.batch_problems(n=n, edges=edges, photmaxes=photmaxes)
    items = []
    for pr in probs:
        p = pr["params"]
        tabs = None if pr["grey"] else W.tables_nb(nB=pr["nB"], nQ=8, nT=64, seed=pr["table_seed"])
        T = W.channel_field(p, seed=pr["field_seed"])
        s = api.Solver(p, tabs, device=dev)
        Q = np.zeros(api.result_shape(p), np.float32)
        S = np.zeros(api.result_shape(p), np.float32)
        items.append(dict(p=p, tabs=tabs, T=T, s=s, Q=Q, S=S))
    return items


def leg_batched(dev, passes=2, tol=None, max_bundles=2.5e11, served=True, warm=True, **mix):
    """Plain (one solve per launch, host arrays in and out, one after the
    other) vs batched (every solve in one persistent launch replayed from a
    CUDA graph) vs served (all submitted to the continuous-batching server at
    once) on the uneven mix.  Wall clock per pass of all 64 solves.  With
    `tol`, every problem first runs a pilot at its recipe photmax and then
    uses the photmax that brings the relative standard deviation of its
    max|Q| to tol (it falls as photmax^-1/2): the comparison at equal
    tolerance.  warm=False skips the untimed first pass of each mode (the
    pilots have run every problem once; the batch's graph is captured inside
    its timed pass, which costs well under 1% of a pass at this size)."""
    import math

    from radchan_b200 import api
    items = batch_setup(dev, **mix)
    if tol is not None:
        for it in items:
            r = it["s"].solve(it["T"])
            rel = api.rel_std_maxq(r.q64, np.sqrt(r.var64))
            q = api.copy_params(it["p"])
            q.photmax = int(math.ceil(it["p"].photmax * (rel / tol) ** 2))
            it["s"].close()
            it["p"] = q
            it["s"] = api.Solver(q, it["tabs"], device=dev)
    work = [it["p"].imax * it["p"].jmax * it["p"].kmax * it["p"].nVar * it["p"].photmax for it in items]
    if sum(work) > max_bundles:
        for it in items:
            it["s"].close()
        return {"skipped": "%.3g bundles per pass exceed the leg's bound %.3g" % (sum(work), max_bundles)}
    big = items[int(np.argmax(work))]
    knobs = big["s"].autotune(big["T"], pilot_photmax=min(big["p"].photmax, 128))
    for it in items:
        it["s"].set_launch(*knobs)
    bundles = float(sum(work))

    # ray-cell steps of one pass, read from each solve's info (the mix's
    # problems take very different numbers of steps per bundle, so steps/s
    # is the comparable rate)
    steps_seen = []

    def plain_pass():
        t0 = time.perf_counter()
        n = 0.0
        for it in items:
            t = it["s"].solve_async(it["T"])
            n += it["s"].info(t).steps
            it["s"].collect_into(t, it["Q"], it["S"])
        steps_seen.append(n)
        return time.perf_counter() - t0

    if warm:
        plain_pass()
    t_plain = min(plain_pass() for _ in range(passes))
    steps = steps_seen[-1]
    ref = [it["Q"].copy() for it in items]
    b = api.Batch(device=dev, use_graph=True)
    for it in items:
        b.add(it["s"], it["T"])

    host_collect = []

    def batched_pass():
        t0 = time.perf_counter()
        b.run()
        b.wait()
        t1 = time.perf_counter()
        for i, it in enumerate(items):
            b.collect_into(i, it["Q"], it["S"])
        t2 = time.perf_counter()
        host_collect.append(t2 - t1)
        return t2 - t0

    if warm:
        batched_pass()
    t_batch = min(batched_pass() for _ in range(passes))
    ph = b.phases()
    phases = {"setup_ms": ph[0], "march_ms": ph[1], "tally_and_copies_ms": ph[2],
              "host_collect_ms": 1000 * min(host_collect),
              "note": "device phases of the last batched run (CUDA events in the graph); host_collect is the "
                      "Fortran-layout scatter of all members after the wait"}
    identical = all(np.array_equal(r, it["Q"]) for r, it in zip(ref, items))
    b.close()
    if not served:
        for it in items:
            it["s"].close()
        n = len(items)
        return {"problems": n, "bundles_per_pass": bundles, "tolerance": tol,
                "photmax_range": [min(it["p"].photmax for it in items), max(it["p"].photmax for it in items)],
                "autotuned": {"rays_per_thread": knobs[0], "block_threads": knobs[1], "sort_bands": knobs[2],
                              "occupancy": knobs[3]},
                "plain_solves_per_s": n / t_plain, "batched_solves_per_s": n / t_batch,
                "batched_vs_plain": t_plain / t_batch, "plain_bundles_per_s": bundles / t_plain,
                "batched_bundles_per_s": bundles / t_batch, "steps_per_pass": steps,
                "plain_steps_per_s": steps / t_plain, "batched_steps_per_s": steps / t_batch,
                "batched_phases": phases, "batched_equals_plain": identical,
                "timing": "wall clock per pass of all solves, host arrays in/out, best of %d after one warm-up "
                          "pass" % passes}
    srv = api.Server(device=dev, max_inflight=len(items))

    def served_pass():
        t0 = time.perf_counter()
        ids = [srv.submit(it["p"], it["T"], table_set=-1 if it["tabs"] is None else it["ts"]) for it in items]
        for rid in ids:
            srv.wait(rid)
        return time.perf_counter() - t0

    for it in items:
        if it["tabs"] is not None:
            it["ts"] = srv.add_tables(it["tabs"])
    served_pass()
    t_srv = min(served_pass() for _ in range(passes))
    srv.close()
    for it in items:
        it["s"].close()
    n = len(items)
    return {"problems": n, "bundles_per_pass": bundles, "tolerance": tol,
            "photmax_range": [min(it["p"].photmax for it in items), max(it["p"].photmax for it in items)],
            "autotuned": {"rays_per_thread": knobs[0], "block_threads": knobs[1], "sort_bands": knobs[2],
                          "occupancy": knobs[3]},
            "plain_solves_per_s": n / t_plain, "batched_solves_per_s": n / t_batch, "served_solves_per_s": n / t_srv,
            "batched_vs_plain": t_plain / t_batch, "served_vs_plain": t_plain / t_srv,
            "plain_bundles_per_s": bundles / t_plain, "batched_bundles_per_s": bundles / t_batch,
            "steps_per_pass": steps, "steps_per_bundle": steps / bundles,
            "plain_steps_per_s": steps / t_plain, "batched_steps_per_s": steps / t_batch,
            "batched_phases": phases, "batched_equals_plain": identical,
            "timing": "wall clock per pass of all solves, host arrays in/out, "
                      "best of %d" % passes}


def serve_run(dev, n_requests, load, inflight=32, policy="srpt", wall_cap=None, seed=2024):
    """Open-loop serving: Poisson arrivals of narrow-band solve requests
    (100 bands x 8 g) with grids drawn from eight classes log-spaced from
    32^3 to 256x128x128, tolerance drawn log-uniformly from 1% to 5%
    relative std of max|Q| (photmax chosen by the server), fields and tables
    resident, admission by a 150 GB budget.  The arrival rate is `load` x
    the capacity 1 / E[service time alone] of the mix, with the service
    time of every size class measured alone after calibration.  With
    wall_cap (seconds) no request is submitted after that time; the ones
    submitted all complete and are reported."""
    import queue
    import threading

    from radchan_b200 import api
    from radchan_b200 import workloads as W
    rng = np.random.default_rng(seed)
    tabs = W.tables_nb()
    classes = []
    for c in range(8):
        r = c / 7.0
        im = int(round(32 * 8 ** r / 8)) * 8
        jm = int(round(32 * 4 ** r / 8)) * 8
        p = W.channel_params(im, jm, jm, photmax=64, nVar=4, levels=[(im, jm, jm), (im // 2, jm // 2, jm // 2),
                                                                     (im // 4, jm // 4, jm // 4)],
                             maxs=[5, 5, 100000], calcwalls=1, adiabw=1)
        classes.append((p, W.channel_field(p, seed=100 + c)))
    srv = api.Server(device=dev, hbm_budget_bytes=150e9, max_inflight=inflight)
    srv.set_policy(policy)
    ts = srv.add_tables(tabs)
    reqs = []
    for _ in range(n_requests):
        reqs.append((int(rng.integers(0, 8)), float(np.exp(rng.uniform(np.log(0.01), np.log(0.05))))))
    # calibration of every class (pilot + one solve at 3%), then the service
    # time of each class alone at its calibrated photmax (no other request)
    alone = []
    for p, T in classes:
        srv.wait(srv.submit(p, T, table_set=ts, tolerance=0.03))
        r = srv.wait(srv.submit(p, T, table_set=ts, tolerance=0.03))
        alone.append((r.t_done - r.t_admit, r.photmax))
    # capacity: one over the mean service time alone of the request mix
    # (photmax grows as 1/tol^2 from the 3% calibration)
    mean_svc = float(np.mean([alone[c][0] * (0.03 / tol) ** 2 for c, tol in reqs]))
    cap = 1.0 / mean_svc
    rate = load * cap
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    results = []
    pending = queue.Queue()

    def waiter():
        while True:
            item = pending.get()
            if item is None:
                return
            i, rid = item
            results.append((i, srv.wait(rid)))

    th = threading.Thread(target=waiter)
    th.start()
    st0 = srv.stats()
    t0 = time.perf_counter()
    t_next = t0
    n_sub = 0
    for i, (c, tol) in enumerate(reqs):
        t_next += gaps[i]
        if wall_cap is not None and t_next - t0 > wall_cap:
            break
        d = t_next - time.perf_counter()
        if d > 0:
            time.sleep(d)
        pending.put((i, srv.submit(classes[c][0], classes[c][1], table_set=ts, tolerance=tol)))
        n_sub += 1
    pending.put(None)
    th.join()
    wall = time.perf_counter() - t0
    st1 = srv.stats()
    srv.close()
    results.sort(key=lambda x: x[0])
    done = [reqs[i] for i, _ in results]
    res = [r for _, r in results]
    lat = np.array([r.latency for r in res])
    # service time alone, scaled by photmax from the class's calibration solve
    svc = np.array([alone[c][0] * r.photmax / alone[c][1] for r, (c, _) in zip(res, done)])
    slow = lat / svc
    met = np.array([r.rel_std_maxq <= 1.25 * tol for r, (_, tol) in zip(res, done)])
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    per_class = {}
    for c, (p, _) in enumerate(classes):
        m = np.array([cc == c for cc, _ in done], bool)
        if m.any():
            per_class["%dx%dx%d" % (p.imax, p.jmax, p.kmax)] = {
                "requests": int(m.sum()), "p50_s": pct(lat[m], 50), "p99_s": pct(lat[m], 99),
                "p99_over_p50": pct(lat[m], 99) / pct(lat[m], 50), "slowdown_p50": pct(slow[m], 50),
                "slowdown_p99": pct(slow[m], 99), "alone_p50_s": pct(svc[m], 50)}
    return {"requests": len(res), "requests_drawn": len(reqs), "wall_cap_s": wall_cap, "load": load,
            "capacity_solves_per_s": cap, "policy": policy, "offered_solves_per_s": rate,
            "solves_per_s": len(res) / wall, "wall_s": wall,
            "p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "p99_over_p50": pct(lat, 99) / pct(lat, 50),
            "alone_p50_s": pct(svc, 50), "alone_p99_s": pct(svc, 99),
            "alone_p99_over_p50": pct(svc, 99) / pct(svc, 50),
            "slowdown_p50": pct(slow, 50), "slowdown_p99": pct(slow, 99),
            "mean_photmax": float(np.mean([r.photmax for r in res])), "tolerance_met_frac": float(met.mean()),
            "gpu_busy_frac": (st1["busy_s"] - st0["busy_s"]) / wall, "hbm_in_use_gb": st1["hbm_in_use"] / 1e9,
            "per_class": per_class,
            "config": {"workload": "Poisson stream, narrow-band 100x8, grids 32^3..256x128x128 in 8 log-spaced "
                                   "classes, tolerance 1-5% log-uniform, 150 GB budget",
                       "classes": [[p.imax, p.jmax, p.kmax] for p, _ in classes], "max_inflight": inflight}}


def run_serve(args, rank, local):
    """--serve: the serving run alone (no wall cap unless --serve-cap)."""
    if rank != 0:
        return
    out = serve_run(local, args.serve_requests, args.load, args.serve_inflight, args.policy, args.serve_cap)
    line = dict({"metric": "serve latency p50/p99 and solves/s", "impl": "ours", "n_gpus": 1, "data": "synthetic"},
                **out)
    print(json.dumps(line), flush=True)


def run_precision(args, rank, local):
    """Precision study: 192x128x128, optically thick tables (log10 k0 in
    [-1, 2]), emissivity 0.8, specular y walls, adiabatic x walls with wall
    fluxes, photmax 1024, nVar 8.  The FP32 march with FP64 tally against the
    full-FP64 build with identical Philox streams; per-cell and wall-flux
    differences in units of the Monte Carlo standard deviation."""
    if rank != 0:
        return
    from radchan_b200 import api
    from radchan_b200 import workloads as W
    tabs = W.tables_nb(logk_lo=-1.0, logk_hi=2.0)
    p32 = W.config_precision(photmax=args.photmax or 1024)
    p64 = api.copy_params(p32)
    p64.floatpoint = 1
    T = W.channel_field(p32, seed=11)
    out = {}
    res = {}
    for name, p in (("fp32", p32), ("fp64", p64)):
        s = api.Solver(p, tabs, device=local)
        t = s.solve_async(T)
        info = s.info(t)
        res[name] = s.collect(t)
        out[name] = {"ms_solve": info.ms_solve, "bundles_per_s": info.bundles / (info.ms_solve / 1000.0),
                     "rel_std_maxq": api.rel_std_maxq(res[name].q64, np.sqrt(res[name].var64))}
        s.close()
    line = {"metric": "FP32 march vs FP64 build, error in MC standard deviations", "impl": "ours", "n_gpus": 1,
            "data": "synthetic", "runs": out, "error_in_sigma": api.compare_in_sigma(res["fp32"], res["fp64"]),
            "fp64_over_fp32_time": out["fp64"]["ms_solve"] / out["fp32"]["ms_solve"],
            "config": {"workload": "192x128x128 narrow-band 100x8, log10 k0 in [-1,2], eps 0.8, specular y, "
                                   "adiabatic x walls with fluxes, photmax %d, nVar 8" % p32.photmax}}
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch

    from radchan_b200 import api
    p, tabs, T, desc = workload(args.workload, args.photmax)
    dev = local
    torch.cuda.set_device(dev)
    s = api.Solver(p, tabs, device=dev)
    if args.rays_per_thread or args.block or args.occupancy or args.sort >= 0:
        s.set_launch(rays_per_thread=args.rays_per_thread, block_threads=args.block, sort_bands=args.sort,
                     occupancy=args.occupancy)
    if args.prio is not None:
        s.set_priority(args.prio)
    T_dev = torch.from_numpy(T).to(f"cuda:{dev}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    # k_init_scalars, k_tmax, k_setup1, k_setup2, k_levels, k_patch_desc,
    # k_march, k_tally (+ k_grey_ib, k_build_ki for a grey gas); the
    # long-ray priority list (k_prio_tiles) is built by the first warm-up
    # solve and reused, as it does not depend on the field
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
            rel_std = api.rel_std_maxq(r.q64, np.sqrt(r.var64))
        else:
            s.release(t)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    barrier(ws)
    t_dev = sum(ms_solve) / 1000.0
    t_max = allreduce_max(t_dev, ws)
    value = bundles * ws / t_max  # == replica_value(bundles, t_dev, ws)
    # e2e through the public API with host buffers: every step copies its
    # field in and its result out; the next solve is issued before the
    # previous one is collected (a context has two solve slots), so the
    # host copies overlap the other slot's solve
    Qh = np.zeros(api.result_shape(p), np.float32)
    Sh = np.zeros(api.result_shape(p), np.float32)

    def e2e_run(n):
        pending = s.solve_async(T)
        for k in range(n):
            nxt = s.solve_async(T) if k + 1 < n else None
            s.collect_into(pending, Qh, Sh)
            pending = nxt

    e2e_run(max(1, args.warmup))
    barrier(ws)
    t0 = time.perf_counter()
    e2e_run(args.steps)
    t_e2e = allreduce_max(time.perf_counter() - t0, ws)
    kl = p.kmax // p.p_col
    d2h = (2 * p.imax * p.jmax * kl + 4 * p.jmax * kl) * 4
    e2e = {"value": bundles * ws / t_e2e, "unit": "bundles/s", "h2d_bytes_per_step": int(T.nbytes),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": 1000 * t_e2e / args.steps, "solves_in_flight": 2}
    peak, peak_kind = peaks()
    march_s = sum(ms_march) / 1000.0
    achieved = steps * 32.0 / march_s / 1e9
    traffic = args.traffic if args.traffic is not None else K_MARCH_TRAFFIC.get(args.workload)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": "k_march", "peak_source": peak_kind,
            "algorithmic_bytes_per_step": 32, "steps_per_launch": steps / args.steps}
    roof.update(gather_ceilings(p, achieved, dev))
    line = {"metric": BUNDLE_METRIC, "value": value, "unit": "bundles/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(desc, ws),
            "steps_per_s": steps * ws / t_max, "solves_per_s": args.steps * ws / t_max,
            "rel_std_maxq": rel_std, "march_ms": 1000 * march_s / args.steps,
            "roofline": roof, "e2e": e2e, "gpu_launches": kernels_per_solve * args.steps,
            "clocks": clk, "wall_s": wall}
    if ws == 1 and not args.no_legs:
        line["at_1pct"] = leg_at_tolerance(p, tabs, T, rel_std, dev, flush)
        line["batched"] = leg_batched(dev)
        # the same recipe restricted to small problems (edges 16-32, photmax
        # 32/128), where one solve does not fill the GPU
        line["batched_small"] = leg_batched(dev, edges=(16, 24, 32), photmaxes=(32, 128))
        line["dns_source"] = leg_dns_source(dev, flush, cpu=not args.no_cpu_baseline)
        # the same solve in a medium with scattering particles
        line["scattering"] = leg_scattering(p, tabs, T, dev, flush)
        # the same mixes at equal 1% relative std of max|Q| (photmax per
        # problem from a pilot), one pass each
        line["batched_at_1pct"] = leg_batched(dev, passes=1, tol=0.01, served=False, warm=False)
        line["batched_small_at_1pct"] = leg_batched(dev, passes=1, tol=0.01, served=False, warm=False,
                                                    edges=(16, 24, 32), photmaxes=(32, 128))
        # serving: the open-loop Poisson stream at 80% load, bounded in wall
        # time (requests submitted within the cap all complete)
        line["serve"] = serve_run(dev, 200, 0.8, wall_cap=args.serve_leg_cap)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
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
    ap.add_argument("--sort", type=int, default=-1, help="band-sorted bundle order 0/1 (default: context's)")
    ap.add_argument("--prio", type=float, default=None,
                    help="long-ray priority: path-length threshold in channel widths (0: off; default: context's)")
    ap.add_argument("--ref-seconds", dest="ref_seconds", type=float, default=12.0)
    ap.add_argument("--traffic", type=float, default=None)
    ap.add_argument("--photmax", type=int, default=0, help="override bundles per cell (profiling runs)")
    ap.add_argument("--no-cpu-baseline", dest="no_cpu_baseline", action="store_true")
    ap.add_argument("--no-legs", dest="no_legs", action="store_true",
                    help="skip the 1%%-tolerance and batched-mix legs (profiling runs)")
    ap.add_argument("--serve", action="store_true", help="open-loop serving run instead of the solve benchmark")
    ap.add_argument("--precision", action="store_true", help="FP32 march vs FP64 build study instead")
    ap.add_argument("--scatter-leg", dest="scatter_leg", action="store_true",
                    help="only the particle-scattering leg (profiling runs; --photmax applies)")
    ap.add_argument("--dns-leg", dest="dns_leg", action="store_true",
                    help="only the DNS coupling leg (profiling runs)")
    ap.add_argument("--serve-requests", dest="serve_requests", type=int, default=200)
    ap.add_argument("--serve-inflight", dest="serve_inflight", type=int, default=32)
    ap.add_argument("--serve-leg-cap", dest="serve_leg_cap", type=float, default=60.0,
                    help="wall-time cap of the default run's serving leg (s)")
    ap.add_argument("--serve-cap", dest="serve_cap", type=float, default=None,
                    help="no new request after this many seconds (serving run)")
    ap.add_argument("--policy", default="srpt", choices=["srpt", "fair"])
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--ref-cuda-child", dest="ref_cuda_child", nargs=3, default=None,
                    help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ref_cuda_child:
        lib, out, ph = args.ref_cuda_child
        ref_cuda_child(lib, out, int(ph))
        return
    ws, rank, local = dist_init()
    if args.serve:
        run_serve(args, rank, local)
    elif args.precision:
        run_precision(args, rank, local)
    elif args.scatter_leg:
        import torch
        torch.cuda.set_device(local)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:%d" % local)
        p, tabs, T, _ = workload(args.workload, args.photmax)
        leg = leg_scattering(p, tabs, T, local, flush, steps=args.steps)
        if rank == 0:
            print(json.dumps(leg), flush=True)
    elif args.dns_leg:
        import torch
        torch.cuda.set_device(local)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:%d" % local)
        leg = leg_dns_source(local, flush, reps=args.steps, cpu=not args.no_cpu_baseline)
        if rank == 0:
            print(json.dumps(leg), flush=True)
    elif args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
