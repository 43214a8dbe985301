"""One solve spread over the ranks of a torch.distributed process group.

The reference splits a solve over GPUs and nodes by slabs of emitting cells
while every GPU holds the whole temperature field (src/montecarlo/
mc_gpu_noint.cu:97-98: z slabs of kmax/p_col planes per node, `zstart`), and
the DNS sums the slabs' results with an MPI_Allreduce (src/dns/fixvar.f:
202-203).  Here rank r of a group of N solves the z slab
k = r*kmax/N + 1 .. (r+1)*kmax/N of the field that rank 0 broadcasts, and
the slabs' results are all-gathered, so every rank ends with the whole
solution.  Bundles are drawn from counters of the global cell index, so the
gathered result equals the same problem solved on one GPU, bit for bit.

With the NCCL backend the field is broadcast into device memory, solved
from there (rc_solve_device_async) and the results are gathered from
device arrays (rc_collect_device); with gloo (CPU tensors) the same steps go
through host arrays.  There is no other data-path collective.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import api


@dataclass
class ShardedResult:
    q64: np.ndarray    # [kmax, jmax, imax] per-cell mean (FP64)
    var64: np.ndarray  # variance of the mean
    qw64: np.ndarray   # [2, kmax, jmax] wall fluxes (west, east)
    vw64: np.ndarray

    def fortran(self, p):
        """Q and sigma in the layout get_results_ fills for a one-slab
        solve: (kmax+2, jmax+2, imax+2) float32, walls at i = 0 / imax+1
        where their flux is computed (mc_gpu_noint.cu:975-1005)."""
        Q = np.zeros((p.kmax + 2, p.jmax + 2, p.imax + 2), np.float32)
        S = np.zeros_like(Q)
        Q[1:-1, 1:-1, 1:-1] = self.q64.astype(np.float32)
        S[1:-1, 1:-1, 1:-1] = np.sqrt(self.var64).astype(np.float32)
        if p.adiabw or p.adiabe:
            for w, i, on in ((0, 0, p.calcwalls and p.adiabw), (1, p.imax + 1, p.calcwalls and p.adiabe)):
                Q[1:-1, 1:-1, i] = self.qw64[w].astype(np.float32) if on else 0.0
                S[1:-1, 1:-1, i] = np.sqrt(self.vw64[w]).astype(np.float32) if on else 0.0
        return Q, S


def slab(kmax, world, rank):
    """(kloc, zstart) of rank `rank` in a group of `world` (mc_gpu_noint.cu:97)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a group of %d" % (rank, world))
    if kmax % world:
        raise ValueError("kmax = %d is not a multiple of the group size %d" % (kmax, world))
    kloc = kmax // world
    return kloc, rank * kloc + 1


class ShardedSolver:
    """A solver context per rank for its z slab of one problem.

    solver_factory(params, tables, device) builds the per-rank solver (the
    default is api.Solver); params.p_col is set to the group size."""

    def __init__(self, params, tables=None, group=None, device=None, solver_factory=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.p = api.copy_params(params)
        self.kloc, self.zstart = slab(self.p.kmax, self.world, self.rank)
        self.p.p_col = self.world
        self.nccl = dist.get_backend(group) == "nccl"
        if self.nccl:
            self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        else:
            self.device = torch.device("cpu")
        dev_index = self.device.index if self.nccl else (0 if device is None else device)
        self.solver = (solver_factory or api.Solver)(self.p, tables, dev_index)

    def solve(self, T=None) -> ShardedResult:
        """T: the whole field (kmax+2, jmax+2, imax+2) float32 on rank 0
        (ignored elsewhere).  Returns the whole solution on every rank."""
        import torch
        p = self.p
        shape = api.field_shape(p)
        if self.rank == 0:
            T = np.ascontiguousarray(T, dtype=np.float32)
            if T.shape != shape:
                raise ValueError("T has shape %s, expected %s" % (T.shape, shape))
            Tt = torch.from_numpy(T).to(self.device)
        else:
            Tt = torch.empty(shape, dtype=torch.float32, device=self.device)
        self.dist.broadcast(Tt, src=0, group=self.group)
        kl, jm, im = self.kloc, p.jmax, p.imax
        f64 = dict(dtype=torch.float64, device=self.device)
        q, v = torch.empty((kl, jm, im), **f64), torch.empty((kl, jm, im), **f64)
        qw, vw = torch.empty((2, kl, jm), **f64), torch.empty((2, kl, jm), **f64)
        if self.nccl:
            t = self.solver.solve_device_async(Tt.data_ptr(), zstart=self.zstart)
            self.solver.collect_device(t, q.data_ptr(), v.data_ptr(), qw.data_ptr(), vw.data_ptr())
        else:
            r = self.solver.collect(self.solver.solve_async(Tt.numpy(), zstart=self.zstart))
            for dst, src in ((q, r.q64), (v, r.var64), (qw, r.qw64), (vw, r.vw64)):
                dst.copy_(torch.from_numpy(np.ascontiguousarray(src)))
        out = []
        for a in (q, v):
            full = torch.empty((self.world * kl, jm, im), **f64)
            self.dist.all_gather_into_tensor(full, a, group=self.group)
            out.append(full.cpu().numpy())
        for a in (qw, vw):
            full = torch.empty((self.world * 2, kl, jm), **f64)  # rank-major (rank, wall) blocks
            self.dist.all_gather_into_tensor(full, a, group=self.group)
            full = full.view(self.world, 2, kl, jm).permute(1, 0, 2, 3)
            out.append(full.reshape(2, self.world * kl, jm).cpu().numpy())
        return ShardedResult(*out)

    def close(self):
        self.solver.close()
