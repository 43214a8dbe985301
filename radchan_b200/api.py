"""Python mirror of the solver interface (ctypes over libradchan.so).

Mirrors the reference's operator interface for this path: a parameter set
equivalent to src/param/param.h + NarrowBand.h, spectral tables in the
layout of src/montecarlo/read_tables.cpp, and a solve that takes the whole
temperature field T(0:imax+1, 0:jmax+1, 0:kmax+1) and returns the radiative
source Q and its Monte Carlo standard deviation in the layout of
get_results_ (src/montecarlo/mc_gpu_noint.cu:876).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


def default_params() -> L.RcParams:
    p = L.RcParams()
    L.check(L.lib().rc_params_default(C.byref(p)))
    return p


def params_from_headers(param_h: str, narrowband_h: str | None = None) -> L.RcParams:
    p = L.RcParams()
    L.check(L.lib().rc_params_from_headers(param_h.encode(), narrowband_h.encode() if narrowband_h else None,
                                           C.byref(p)))
    return p


def validate(p: L.RcParams) -> str:
    buf = C.create_string_buffer(512)
    rc = L.lib().rc_params_validate(C.byref(p), buf, 512)
    return "" if rc == 0 else buf.value.decode()


def set_levels(p: L.RcParams, levels, maxs):
    """levels: list of (im, jm, km), finest first; maxs: step budgets."""
    p.grid_num = len(levels)
    for l, (a, b, c) in enumerate(levels):
        p.maxi[l], p.maxj[l], p.maxk[l] = a, b, c
        p.maxs[l] = maxs[l]
    return p


def copy_params(p: L.RcParams) -> L.RcParams:
    q = L.RcParams()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(L.RcParams))
    return q


def grid_level(p: L.RcParams, level: int = 0):
    im, jm, km = p.maxi[level], p.maxj[level], p.maxk[level]
    arrs = {n: np.zeros(s, np.float32) for n, s in
            (("xu", im + 1), ("yu", jm + 1), ("zu", km + 1), ("x", im + 2), ("y", jm + 2), ("z", km + 2))}
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    L.check(L.lib().rc_grid_level(C.byref(p), level, fp(arrs["xu"]), fp(arrs["yu"]), fp(arrs["zu"]),
                                  fp(arrs["x"]), fp(arrs["y"]), fp(arrs["z"])))
    return arrs


class TableSet:
    """Host-owned spectral table set (correlated-k tables)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self.view = L.RcTables()
        L.check(L.lib().rc_tables_view(self.h, C.byref(self.view)))

    @classmethod
    def synthetic(cls, nB=100, nQ=8, nT=64, T_lo=300.0, T_hi=2000.0, nu_lo=500.0, nu_hi=10000.0,
                  logk_lo=-3.0, logk_hi=2.0, nexp=1.0, kexp=1.5, seed=20240601):
        s = L.RcSynthSpec(nB, nQ, nT, T_lo, T_hi, nu_lo, nu_hi, logk_lo, logk_hi, nexp, kexp, seed)
        h = C.c_void_p()
        L.check(L.lib().rc_tables_synthetic(C.byref(s), C.byref(h)))
        return cls(h)

    @classmethod
    def read_dir(cls, path, nT, nB, nQ):
        h = C.c_void_p()
        L.check(L.lib().rc_tables_read_dir(str(path).encode(), nT, nB, nQ, C.byref(h)))
        return cls(h)

    def write_dir(self, path):
        L.check(L.lib().rc_tables_write_dir(self.h, str(path).encode()))

    def validate(self) -> str:
        """rc_tables_validate: "" when the set meets the solver's
        assumptions, else the first violation."""
        buf = C.create_string_buffer(512)
        rc = L.lib().rc_tables_validate(C.byref(self.view), buf, 512)
        return "" if rc == L.RC_OK else buf.value.decode(errors="replace")

    def arrays(self):
        v = self.view
        nT, nB, nQ = v.nT, v.nB, v.nQ
        f = lambda ptr, n: np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return dict(nT=nT, nB=nB, nQ=nQ, Tnb=f(v.Tnb, nT), kP=f(v.kP, nT), wvl=f(v.wvl, nB), wvr=f(v.wvr, nB),
                    wvc=f(v.wvc, nB), kavg=f(v.kavg, nB), kq=f(v.kq, nB * nT * nQ).reshape(nB, nT, nQ),
                    prob=f(v.prob, nT * nB).reshape(nT, nB), probg=f(v.probg, nT * nB * nQ).reshape(nT, nB, nQ),
                    wq=f(v.wq, nQ))

    def __del__(self):
        try:
            if self.h:
                L.lib().rc_tables_free(self.h)
                self.h = None
        except Exception:
            pass


class Scattering:
    """Particle scattering tables (rc_scattering): scattering coefficient per
    band and g point, phase-function CDF per band over nA angles.  Either
    host-owned by the library (synthetic, read_dir) or built from numpy
    arrays (from_arrays)."""

    def __init__(self, handle=None, arrays=None):
        self.h = None
        self._keep = None
        if handle is not None:
            self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
            self.view = L.RcScattering()
            L.check(L.lib().rc_scattering_view(self.h, C.byref(self.view)))
        else:
            ksca, theta, cdf, kabs = arrays
            self._keep = [np.ascontiguousarray(a, np.float32) for a in (ksca, theta, cdf)]
            self._keep.append(None if kabs is None else np.ascontiguousarray(kabs, np.float32))
            k, th, cd, ka = self._keep
            fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
            self.view = L.RcScattering(k.shape[0], k.shape[1], th.shape[0], fp(k), fp(ka), fp(th), fp(cd))

    @classmethod
    def from_arrays(cls, ksca, theta, phase_cdf, kabs=None):
        """ksca [nB, nQ] (1/m), theta [nA] radians, phase_cdf [nB, nA]."""
        ksca = np.asarray(ksca, np.float32)
        phase_cdf = np.asarray(phase_cdf, np.float32)
        assert ksca.ndim == 2 and phase_cdf.ndim == 2 and phase_cdf.shape[0] == ksca.shape[0]
        assert phase_cdf.shape[1] == len(theta)
        return cls(arrays=(ksca, theta, phase_cdf, kabs))

    @classmethod
    def synthetic(cls, nB, nQ=1, nA=181, ksca_lo=0.5, ksca_hi=0.5, g_lo=0.0, g_hi=0.0, seed=77):
        s = L.RcScatterSpec(nB, nQ, nA, ksca_lo, ksca_hi, g_lo, g_hi, seed)
        h = C.c_void_p()
        L.check(L.lib().rc_scattering_synthetic(C.byref(s), C.byref(h)))
        return cls(handle=h)

    @classmethod
    def read_dir(cls, path, nB, nQ):
        h = C.c_void_p()
        L.check(L.lib().rc_scattering_read_dir(str(path).encode(), nB, nQ, C.byref(h)))
        return cls(handle=h)

    def write_dir(self, path):
        assert self.h is not None, "only library-owned particle tables are written"
        L.check(L.lib().rc_scattering_write_dir(self.h, str(path).encode()))

    def validate(self) -> str:
        buf = C.create_string_buffer(512)
        rc = L.lib().rc_scattering_validate(C.byref(self.view), buf, 512)
        return "" if rc == L.RC_OK else buf.value.decode(errors="replace")

    def arrays(self):
        v = self.view
        nB, nQ, nA = v.nB, v.nQ, v.nA
        f = lambda ptr, n: np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return dict(nB=nB, nQ=nQ, nA=nA, ksca=f(v.ksca, nB * nQ).reshape(nB, nQ),
                    kabs=f(v.kabs, nB * nQ).reshape(nB, nQ) if v.kabs else None, theta=f(v.theta, nA),
                    phase_cdf=f(v.phase_cdf, nB * nA).reshape(nB, nA))

    def __del__(self):
        try:
            if self.h:
                L.lib().rc_scattering_free(self.h)
                self.h = None
        except Exception:
            pass


def rel_std_maxq(q, sigma):
    """Relative Monte Carlo standard deviation of max|Q|: RMS sigma of the
    cells whose |Q| is within 10% of the maximum, over max|Q| (the
    estimator the server uses to meet a tolerance)."""
    a = np.abs(np.asarray(q, np.float64))
    best = a.max()
    if not best > 0:
        return 0.0
    m = a >= 0.9 * best
    return float(np.sqrt(np.mean(np.asarray(sigma, np.float64)[m] ** 2)) / best)


def compare_in_sigma(a: "Result", b: "Result"):
    """Per-cell and wall-flux differences of two solves of the same problem
    (e.g. the FP32 march and the FP64 build with the same streams) in units
    of the Monte Carlo standard deviation of b."""
    out = {}
    for name, q0, q1, v1 in (("cells", a.q64, b.q64, b.var64), ("walls", a.qw64, b.qw64, b.vw64)):
        q0 = np.asarray(q0, np.float64).ravel()
        q1 = np.asarray(q1, np.float64).ravel()
        s = np.sqrt(np.asarray(v1, np.float64).ravel())
        m = s > 0
        if not m.any():
            continue
        z = (q0[m] - q1[m]) / s[m]
        out[name] = {"n": int(m.sum()), "max_abs_z": float(np.abs(z).max()), "rms_z": float(np.sqrt(np.mean(z * z))),
                     "mean_z": float(z.mean()),
                     "max_rel": float(np.max(np.abs(q0[m] - q1[m]) / np.maximum(np.abs(q1[m]), 1e-300)))}
    return out


def probe_gather(nbytes: int, mode: int = 0, iters: int = 1024, device: int = 0):
    """rc_probe_gather: random 32-byte-sector gather throughput over an
    array of nbytes (mode 0 L2 only, mode 1 through L1); returns (sectors/s,
    GB/s at 32 B per sector, ms of the best launch)."""
    s = C.c_double()
    ms = C.c_float()
    L.check(L.lib().rc_probe_gather(device, int(nbytes), mode, iters, C.byref(s), C.byref(ms)))
    return s.value, s.value * 32 / 1e9, ms.value


def field_shape(p):
    """numpy shape of the temperature field: (kmax+2, jmax+2, imax+2), i fastest."""
    return (p.kmax + 2, p.jmax + 2, p.imax + 2)


def result_shape(p):
    return (p.kmax // p.p_col + 2, p.jmax + 2, p.imax + 2)


@dataclass
class DnsCoupling:
    """How the channel DNS turns a solve into its energy-equation source
    (src/dns/channel.f:249-266, fixvar.f:16-43 and :179-242); see
    rc_dns_coupling in radchan.h."""
    Tin: float                 # temperature scale, K (T = T1 * Tin)
    Height: float              # divides the wall fluxes
    underrelax: float          # multiplies Qnew before Gnew is formed
    Tnb: np.ndarray            # table temperatures, K, uniform step >= 1 K
    kP: np.ndarray             # Planck-mean coefficient times Height
    jstart: int = 1            # 1-based global j range of the DNS pencil
    jend: int = -1             # -1: jmax
    stefan: float = 5.67e-08   # the DNS's constant (src/dns/param.txt:41)

    def struct(self, jmax):
        self._Tnb = np.ascontiguousarray(self.Tnb, np.float64)
        self._kP = np.ascontiguousarray(self.kP, np.float64)
        dp = C.POINTER(C.c_double)
        return L.RcDnsCoupling(self.Tin, self.Height, self.underrelax, self.stefan, len(self._Tnb),
                               self._Tnb.ctypes.data_as(dp), self._kP.ctypes.data_as(dp), self.jstart,
                               jmax if self.jend < 0 else self.jend)

    def pencil_shapes(self, p):
        """(T1 shape, output shape) of the pencil, numpy order (k, j, i)."""
        kl = p.kmax // p.p_col
        jn = (p.jmax if self.jend < 0 else self.jend) - self.jstart + 1
        return (kl + 2, jn + 2, p.imax + 2), (kl, jn, p.imax + 2)


def field_from_dns(T1, Tin):
    """The solver's float field from the DNS's nondimensional double T1
    (whole field with ghosts, numpy order (k, j, i)): real(T1*Tin, 4), the
    conversion of bcastArr (src/dns/routine.f90:205-209).  bcastArr leaves
    the j and k ghost planes of its output untouched; here they come from
    T1's own halo."""
    return (np.asarray(T1, np.float64) * Tin).astype(np.float32)


def read_planck_mean(path, n, height):
    """read_kP (src/dns/fixvar.f:1-14): Tnb and kP * height from the first n
    rows of planck-mean.txt ("T kP kR kM" per row)."""
    rows = []
    with open(path) as f:
        for line in f:
            v = line.split()
            if len(v) >= 2:
                rows.append((float(v[0]), float(v[1])))
            if len(rows) == n:
                break
    if len(rows) < n:
        raise L.RadChanError(-4, "%s has fewer than %d rows" % (path, n))
    a = np.array(rows, np.float64)
    return a[:, 0].copy(), a[:, 1] * height


@dataclass
class Result:
    Q: np.ndarray          # Fortran-layout float result (kloc+2, jmax+2, imax+2)
    sigma: np.ndarray
    q64: np.ndarray        # [kloc, jmax, imax] per-cell mean (FP64)
    var64: np.ndarray      # variance of the mean
    qw64: np.ndarray       # [2, kloc, jmax] wall fluxes (west, east)
    vw64: np.ndarray


class Solver:
    """One solver context on one GPU (rc_create .. rc_destroy)."""

    def __init__(self, params: L.RcParams, tables: TableSet | None = None, device: int = 0):
        self.p = copy_params(params)
        self.ctx = C.c_void_p()
        L.check(L.lib().rc_create(C.byref(self.p), device, C.byref(self.ctx)))
        self.tables = tables
        if tables is not None and not self.p.grey:
            L.check(L.lib().rc_set_tables(self.ctx, C.byref(tables.view)), self.ctx)

    def set_launch(self, rays_per_thread=0, block_threads=0, sort_bands=-1, occupancy=0):
        L.check(L.lib().rc_set_launch(self.ctx, rays_per_thread, block_threads, sort_bands, occupancy), self.ctx)

    def set_scattering(self, sc: "Scattering | None"):
        """rc_set_scattering: particle scattering for later solves (None
        removes it)."""
        self.scattering = sc
        L.check(L.lib().rc_set_scattering(self.ctx, C.byref(sc.view) if sc is not None else None), self.ctx)

    def set_priority(self, threshold: float):
        """rc_set_priority: tiles holding a bundle with |s_x| < threshold
        are marched first (0 turns it off); results do not change."""
        L.check(L.lib().rc_set_priority(self.ctx, float(threshold)), self.ctx)

    def get_launch(self):
        """(rays_per_thread, block_threads, sort_bands, occupancy)"""
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib().rc_get_launch(self.ctx, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), self.ctx)
        return a.value, b.value, c.value, d.value

    def solve_async(self, T: np.ndarray, zstart: int = 1) -> int:
        T = np.ascontiguousarray(T, dtype=np.float32)
        assert T.shape == field_shape(self.p), (T.shape, field_shape(self.p))
        t = C.c_int32()
        L.check(L.lib().rc_solve_async(self.ctx, T.ctypes.data_as(C.POINTER(C.c_float)), zstart, C.byref(t)),
                self.ctx)
        return t.value

    def solve_device_async(self, T_dev_ptr: int, zstart: int = 1) -> int:
        t = C.c_int32()
        L.check(L.lib().rc_solve_device_async(self.ctx, C.c_void_p(T_dev_ptr), zstart, C.byref(t)), self.ctx)
        return t.value

    def collect(self, ticket: int, want64: bool = True) -> Result:
        p = self.p
        kl = p.kmax // p.p_col
        Q = np.zeros(result_shape(p), np.float32)
        S = np.zeros(result_shape(p), np.float32)
        q64 = np.zeros((kl, p.jmax, p.imax)) if want64 else None
        v64 = np.zeros((kl, p.jmax, p.imax)) if want64 else None
        qw = np.zeros((2, kl, p.jmax)) if want64 else None
        vw = np.zeros((2, kl, p.jmax)) if want64 else None
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
        L.check(L.lib().rc_collect(self.ctx, ticket, fp(Q), fp(S), dp(q64), dp(v64), dp(qw), dp(vw)), self.ctx)
        return Result(Q, S, q64, v64, qw, vw)

    def collect_into(self, ticket: int, Q: np.ndarray, S: np.ndarray):
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        L.check(L.lib().rc_collect(self.ctx, ticket, fp(Q), fp(S), None, None, None, None), self.ctx)

    def collect_device(self, ticket: int, q64_dev: int, var64_dev: int = 0, qw64_dev: int = 0, vw64_dev: int = 0):
        """rc_collect_device: the compact double results into device arrays
        (pointers; 0 skips one); the ticket is consumed."""
        v = lambda x: C.c_void_p(x) if x else None
        L.check(L.lib().rc_collect_device(self.ctx, ticket, v(q64_dev), v(var64_dev), v(qw64_dev), v(vw64_dev)),
                self.ctx)

    def wait_device(self, ticket: int):
        q = C.c_void_p()
        L.check(L.lib().rc_device_results(self.ctx, ticket, C.byref(q), None, None, None), self.ctx)
        return q.value

    def release(self, ticket: int):
        L.check(L.lib().rc_collect(self.ctx, ticket, None, None, None, None, None, None), self.ctx)

    def info(self, ticket: int) -> L.RcSolveInfo:
        i = L.RcSolveInfo()
        L.check(L.lib().rc_solve_info_get(self.ctx, ticket, C.byref(i)), self.ctx)
        return i

    def solve(self, T, zstart=1, want64=True) -> Result:
        return self.collect(self.solve_async(T, zstart), want64)

    def dns_source(self, ticket: int, cpl: DnsCoupling, T1: np.ndarray):
        """Wait for a ticket and return the DNS source terms of the pencil
        (rc_dns_source): dict of Qnew, Varnew, Knew, Gnew as (kloc, jn,
        imax+2) float64 arrays and n_clamped.  The ticket is consumed."""
        s = cpl.struct(self.p.jmax)
        tshape, oshape = cpl.pencil_shapes(self.p)
        T1 = np.ascontiguousarray(T1, np.float64)
        assert T1.shape == tshape, (T1.shape, tshape)
        out = {k: np.empty(oshape, np.float64) for k in ("Qnew", "Varnew", "Knew", "Gnew")}
        n = C.c_longlong()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        L.check(L.lib().rc_dns_source(self.ctx, ticket, C.byref(s), dp(T1), dp(out["Qnew"]), dp(out["Varnew"]),
                                      dp(out["Knew"]), dp(out["Gnew"]), C.byref(n)), self.ctx)
        out["n_clamped"] = n.value
        return out

    def dns_source_device(self, ticket: int, cpl: DnsCoupling, T1_dev: int, Qnew_dev: int, Varnew_dev: int,
                          Knew_dev: int, Gnew_dev: int, n_clamped_dev: int = 0, stream: int = 0):
        """rc_dns_source_device: the same on device pointers, enqueued on
        `stream` (0: the solve's stream); returns at once, the ticket stays."""
        s = cpl.struct(self.p.jmax)
        v = lambda x: C.c_void_p(x) if x else None
        L.check(L.lib().rc_dns_source_device(self.ctx, ticket, C.byref(s), v(T1_dev), v(Qnew_dev), v(Varnew_dev),
                                             v(Knew_dev), v(Gnew_dev), v(n_clamped_dev), v(stream)), self.ctx)

    def trace(self, ticket, ids, max_cells=0):
        n = len(ids)
        arr = (L.RcBundleId * n)(*[L.RcBundleId(*b) for b in ids])
        out = (L.RcTraceRec * n)()
        cells = np.full((n, max(max_cells, 1), 4), -1, np.int32)
        L.check(L.lib().rc_trace(self.ctx, ticket, n, arr, out, max_cells,
                                 cells.ctypes.data_as(C.POINTER(C.c_int)) if max_cells > 0 else None), self.ctx)
        return list(out), cells[:, :max_cells]

    def sample_bands(self, ticket, kind, u_band, u_g):
        """Band and g point that emission selects for the given uniforms
        (rc_sample_bands)."""
        ub = np.ascontiguousarray(u_band, np.float32)
        ug = np.ascontiguousarray(u_g, np.float32)
        assert ub.shape == ug.shape and ub.ndim == 1
        nb = np.zeros(ub.size, np.int32)
        g = np.zeros(ub.size, np.int32)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        L.check(L.lib().rc_sample_bands(self.ctx, ticket, kind, ub.size, fp(ub), fp(ug), ip(nb), ip(g)), self.ctx)
        return nb, g

    def autotune(self, T, zstart=1, pilot_photmax=16):
        """Pick rays_per_thread, block_threads, sort_bands and occupancy by
        timing pilot solves on T; returns the chosen (rpt, block, sort, occupancy)."""
        T = np.ascontiguousarray(T, dtype=np.float32)
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib().rc_autotune(self.ctx, T.ctypes.data_as(C.POINTER(C.c_float)), zstart, pilot_photmax,
                                    C.byref(a), C.byref(b), C.byref(c), C.byref(d)), self.ctx)
        return a.value, b.value, c.value, d.value

    def close(self):
        if self.ctx:
            L.lib().rc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def slab_range(kmax: int, nranks: int, rank: int):
    """rc_slab_range: (kloc, zstart) of rank `rank` in a group of `nranks`."""
    kl, zs = C.c_int(), C.c_int()
    L.check(L.lib().rc_slab_range(kmax, nranks, rank, C.byref(kl), C.byref(zs)))
    return kl.value, zs.value


def slab_unique_id() -> bytes:
    """rc_slab_unique_id: a new group id (RC_SLAB_ID_BYTES bytes) for
    SlabComm; made on one rank and handed to the others."""
    buf = C.create_string_buffer(128)
    L.check_slab(L.lib().rc_slab_unique_id(buf))
    return buf.raw


class SlabComm:
    """One rank of a group that solves problems by z slabs over NCCL from
    the library itself (rc_slab_comm_create .. rc_slab_comm_destroy): the
    C route to what ShardedSolver does over torch.distributed."""

    def __init__(self, device: int, nranks: int, rank: int, uid: bytes, timeout_s: float = 300.0):
        if len(uid) != 128:
            raise ValueError("a group id has 128 bytes")
        self.comm = C.c_void_p()
        L.check_slab(L.lib().rc_slab_comm_create(device, nranks, rank, uid, float(timeout_s), C.byref(self.comm)))
        self.nranks, self.rank = nranks, rank

    def solve(self, solver: "Solver", T: int, q64: int, var64: int, qw64: int = 0, vw64: int = 0):
        """rc_slab_solve with pointers to device or host arrays (0 skips a
        wall output): the whole solution on every rank."""
        v = lambda x: C.c_void_p(x) if x else None
        L.check_slab(L.lib().rc_slab_solve(self.comm, solver.ctx, v(T), v(q64), v(var64), v(qw64), v(vw64)),
                     self.comm)

    def solve_arrays(self, solver: "Solver", T=None):
        """rc_slab_solve with numpy arrays in host memory: T the whole field
        (read on rank 0); returns (q64, var64, qw64, vw64) of the whole
        problem."""
        p = solver.p
        shape = field_shape(p)
        T = np.zeros(shape, np.float32) if T is None else np.ascontiguousarray(T, dtype=np.float32).copy()
        if T.shape != shape:
            raise ValueError("T has shape %s, expected %s" % (T.shape, shape))
        q = np.empty((p.kmax, p.jmax, p.imax))
        v = np.empty_like(q)
        qw = np.empty((2, p.kmax, p.jmax))
        vw = np.empty_like(qw)
        self.solve(solver, T.ctypes.data, q.ctypes.data, v.ctypes.data, qw.ctypes.data, vw.ctypes.data)
        return q, v, qw, vw

    def close(self):
        if self.comm:
            L.check_slab(L.lib().rc_slab_comm_destroy(self.comm))
            self.comm = None


class Batch:
    """Many solves of uneven size in one persistent launch (rc_batch_*)."""

    def __init__(self, device=0, use_graph=True):
        self.h = C.c_void_p()
        L.check(L.lib().rc_batch_create(device, 1 if use_graph else 0, C.byref(self.h)))
        self.members = []

    def add(self, solver: Solver, T: np.ndarray, zstart: int = 1):
        T = np.ascontiguousarray(T, dtype=np.float32)
        self.members.append((solver, T))
        L.check(L.lib().rc_batch_add(self.h, solver.ctx, T.ctypes.data_as(C.POINTER(C.c_float)), zstart))

    def run(self):
        L.check(L.lib().rc_batch_run(self.h))

    def wait(self) -> float:
        ms = C.c_float()
        L.check(L.lib().rc_batch_wait(self.h, C.byref(ms)))
        return ms.value

    def phases(self):
        """Device ms of the last run: (set-up, march, tally + copies)."""
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        L.check(L.lib().rc_batch_phases(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def collect(self, index, want64=True) -> Result:
        s, _ = self.members[index]
        p = s.p
        kl = p.kmax // p.p_col
        Q = np.zeros(result_shape(p), np.float32)
        S = np.zeros(result_shape(p), np.float32)
        q64 = np.zeros((kl, p.jmax, p.imax)) if want64 else None
        v64 = np.zeros((kl, p.jmax, p.imax)) if want64 else None
        qw = np.zeros((2, kl, p.jmax)) if want64 else None
        vw = np.zeros((2, kl, p.jmax)) if want64 else None
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
        L.check(L.lib().rc_batch_collect(self.h, index, fp(Q), fp(S), dp(q64), dp(v64), dp(qw), dp(vw)))
        return Result(Q, S, q64, v64, qw, vw)

    def collect_into(self, index, Q: np.ndarray, S: np.ndarray):
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        L.check(L.lib().rc_batch_collect(self.h, index, fp(Q), fp(S), None, None, None, None))

    def close(self):
        if self.h:
            L.lib().rc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ServedResult:
    Q: np.ndarray          # Fortran-layout float result (kloc+2, jmax+2, imax+2)
    sigma: np.ndarray
    t_submit: float        # seconds on the server's steady clock
    t_admit: float
    t_done: float
    photmax: int           # bundles per cell the solve used
    rel_std_maxq: float    # sigma / |Q| at the cell of max |Q|

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    """Continuous-batching solve server on one GPU (rc_server_*).

    submit() copies the request and returns at once; wait() blocks until the
    request's result is ready.  Requests run concurrently, sharing every
    march launch; each result equals the same request solved alone."""

    def __init__(self, device=0, hbm_budget_bytes=150e9, max_inflight=8):
        self.h = C.c_void_p()
        L.check(L.lib().rc_server_create(device, float(hbm_budget_bytes), max_inflight, C.byref(self.h)))
        self._params = {}
        self._tables = []

    def add_tables(self, tables: TableSet) -> int:
        ts = C.c_int()
        L.check(L.lib().rc_server_add_tables(self.h, C.byref(tables.view), C.byref(ts)))
        self._tables.append(tables)
        return ts.value

    def set_scattering(self, table_set: int, sc: "Scattering | None"):
        """rc_server_set_scattering: particles for the later requests of a
        table set (-1: grey requests); None removes them."""
        self._scatter = getattr(self, "_scatter", {})
        self._scatter[table_set] = sc
        L.check(L.lib().rc_server_set_scattering(self.h, table_set, C.byref(sc.view) if sc is not None else None))

    def submit(self, params: L.RcParams, T: np.ndarray, table_set: int = -1, zstart: int = 1,
               tolerance: float = 0.0) -> int:
        p = copy_params(params)
        T = np.ascontiguousarray(T, dtype=np.float32)
        if T.shape != field_shape(p):
            raise ValueError("T must have shape %s" % (field_shape(p),))
        req = L.RcRequest(C.pointer(p), table_set, T.ctypes.data_as(C.POINTER(C.c_float)), zstart, tolerance)
        rid = C.c_int64()
        L.check(L.lib().rc_server_submit(self.h, C.byref(req), C.byref(rid)))
        self._params[rid.value] = p
        return rid.value

    def wait(self, rid: int) -> ServedResult:
        p = self._params.pop(rid)
        Q = np.zeros(result_shape(p), np.float32)
        S = np.zeros(result_shape(p), np.float32)
        info = L.RcResultInfo()
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        L.check(L.lib().rc_server_wait(self.h, rid, fp(Q), fp(S), C.byref(info)))
        return ServedResult(Q, S, info.t_submit, info.t_admit, info.t_done, info.photmax, info.rel_std_maxq)

    def cancel(self, rid: int):
        """rc_server_cancel: wait(rid) then raises RC_E_CANCELLED, unless
        the solve completed first."""
        L.check(L.lib().rc_server_cancel(self.h, int(rid)))

    def set_quantum(self, tiles: int):
        L.check(L.lib().rc_server_set_quantum(self.h, int(tiles)))

    def set_policy(self, policy: str):
        """'srpt' (least remaining work first, default) or 'fair' (equal shares)."""
        L.check(L.lib().rc_server_set_policy(self.h, {"fair": 0, "srpt": 1}[policy]))

    def stats(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        L.check(L.lib().rc_server_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        q = C.c_longlong()
        L.check(L.lib().rc_server_quanta(self.h, C.byref(q)))
        return {"solves": a.value, "busy_s": b.value, "hbm_in_use": c.value, "quanta": q.value}

    def close(self):
        if self.h:
            L.lib().rc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
