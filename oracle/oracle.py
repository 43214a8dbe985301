"""ctypes bindings of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs, never by the product package.  It does not import the
product package either: the C structures come from oracle/abi.py.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from oracle import abi as L

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


class OracleSetup(C.Structure):
    _fields_ = [("Tmax", C.c_float), ("Tmin", C.c_float), ("tm", C.c_int), ("row", C.c_int), ("status", C.c_int),
                ("kappamax", C.c_double), ("Ibmax_f", C.c_double), ("Ibmax_w", C.c_double * 2),
                ("T0", C.c_double), ("inv_dT", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from oracle import build as _b
            _b.build()
        L_ = C.CDLL(LIB_PATH)
        PP = C.POINTER(L.RcParams)
        TP = C.POINTER(L.RcTables)
        FP = C.POINTER(C.c_float)
        DP = C.POINTER(C.c_double)
        L_.oracle_solve.restype = C.c_int
        L_.oracle_solve.argtypes = [PP, TP, FP, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_int, C.c_int,
                                    C.c_int, DP, DP, DP, DP, DP, DP]
        L_.oracle_trace.restype = C.c_int
        L_.oracle_trace.argtypes = [PP, TP, FP, C.c_int, C.c_int, C.c_int, C.POINTER(L.RcBundleId),
                                    C.POINTER(L.RcTraceRec), C.c_int, C.POINTER(C.c_int)]
        L_.oracle_setup_scalars.restype = C.c_int
        L_.oracle_setup_scalars.argtypes = [PP, TP, FP, C.c_int, C.POINTER(OracleSetup)]
        L_.oracle_grid_level.restype = C.c_int
        L_.oracle_grid_level.argtypes = [PP, C.c_int, FP, FP, FP, FP, FP, FP]
        L_.oracle_level_T.restype = C.c_int
        L_.oracle_level_T.argtypes = [PP, FP, C.c_int, FP]
        _lib = L_
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _tv(tables):
    return C.byref(L.tables_view(tables.view)) if tables is not None else None


def _pp(p):
    return C.byref(L.params(p))


class _Scattering:
    """Holds the arrays of particle scattering tables while the oracle
    solves with them: ksca [nB, nQ], theta [nA] (radians), phase_cdf
    [nB, nA]."""

    def __init__(self, ksca, theta, phase_cdf):
        self.k = np.ascontiguousarray(ksca, np.float32)
        self.t = np.ascontiguousarray(theta, np.float32)
        self.c = np.ascontiguousarray(phase_cdf, np.float32)
        nB, nQ = self.k.shape
        self.s = L.RcScattering(nB, nQ, self.t.shape[0], _fp(self.k), None, _fp(self.t), _fp(self.c))


class scattering:
    """Context manager: the oracle's solves and traces inside it see the
    given particle scattering tables (an object with ksca, theta, phase_cdf
    arrays, or a dict with those keys); None means none."""

    def __init__(self, sc):
        self.sc = sc

    def __enter__(self):
        if self.sc is not None:
            g = (lambda k: self.sc[k]) if isinstance(self.sc, dict) else (lambda k: getattr(self.sc, k))
            self.h = _Scattering(g("ksca"), g("theta"), g("phase_cdf"))
            f = lib().oracle_set_scattering
            f.restype = C.c_int
            f.argtypes = [C.POINTER(L.RcScattering)]
            if f(C.byref(self.h.s)) != 0:
                raise RuntimeError("oracle_set_scattering failed")
        return self

    def __exit__(self, *a):
        f = lib().oracle_set_scattering
        f.restype = C.c_int
        f.argtypes = [C.POINTER(L.RcScattering)]
        f(None)
        return False


def solve(p, tables, T, zstart=1, rpt=8, cell_begin=0, cell_end=-1, walls=True, fp64=False, nthreads=0,
          scatter=None):
    if scatter is not None:
        with scattering(scatter):
            return solve(p, tables, T, zstart, rpt, cell_begin, cell_end, walls, fp64, nthreads)
    T = np.ascontiguousarray(T, dtype=np.float32)
    kl = p.kmax // p.p_col
    q = np.full((kl, p.jmax, p.imax), np.nan)
    v = np.full((kl, p.jmax, p.imax), np.nan)
    qw = np.zeros((2, kl, p.jmax))
    vw = np.zeros((2, kl, p.jmax))
    st = C.c_double()
    nb = C.c_double()
    rc = lib().oracle_solve(_pp(p), _tv(tables), _fp(T), zstart, rpt, cell_begin, cell_end, 1 if walls else 0,
                            1 if fp64 else 0, nthreads, _dp(q), _dp(v), _dp(qw), _dp(vw), C.byref(st), C.byref(nb))
    if rc != 0:
        raise RuntimeError("oracle_solve failed: %d" % rc)
    return dict(q64=q, var64=v, qw64=qw, vw64=vw, steps=st.value, bundles=nb.value)


def trace(p, tables, T, ids, max_cells=0, fp64=False, scatter=None):
    if scatter is not None:
        with scattering(scatter):
            return trace(p, tables, T, ids, max_cells, fp64)
    T = np.ascontiguousarray(T, dtype=np.float32)
    n = len(ids)
    arr = (L.RcBundleId * n)(*[L.RcBundleId(*b) for b in ids])
    out = (L.RcTraceRec * n)()
    cells = np.full((n, max(max_cells, 1), 4), -1, np.int32)
    rc = lib().oracle_trace(_pp(p), _tv(tables), _fp(T), 1, 1 if fp64 else 0, n, arr, out, max_cells,
                            cells.ctypes.data_as(C.POINTER(C.c_int)) if max_cells > 0 else None)
    if rc != 0:
        raise RuntimeError("oracle_trace failed: %d" % rc)
    return list(out), cells[:, :max_cells]


def setup(p, tables, T, fp64=False):
    T = np.ascontiguousarray(T, dtype=np.float32)
    s = OracleSetup()
    rc = lib().oracle_setup_scalars(_pp(p), _tv(tables), _fp(T), 1 if fp64 else 0, C.byref(s))
    if rc != 0:
        raise RuntimeError("oracle_setup_scalars failed: %d" % rc)
    return s


def grid_level(p, level=0):
    im, jm, km = p.maxi[level], p.maxj[level], p.maxk[level]
    a = {n: np.zeros(s, np.float32) for n, s in
         (("xu", im + 1), ("yu", jm + 1), ("zu", km + 1), ("x", im + 2), ("y", jm + 2), ("z", km + 2))}
    rc = lib().oracle_grid_level(_pp(p), level, _fp(a["xu"]), _fp(a["yu"]), _fp(a["zu"]), _fp(a["x"]),
                                 _fp(a["y"]), _fp(a["z"]))
    if rc != 0:
        raise RuntimeError("oracle_grid_level failed")
    return a


def level_T(p, T, level):
    T = np.ascontiguousarray(T, dtype=np.float32)
    out = np.zeros((p.maxk[level], p.maxj[level], p.maxi[level]), np.float32)
    rc = lib().oracle_level_T(_pp(p), _fp(T), level, _fp(out))
    if rc != 0:
        raise RuntimeError("oracle_level_T failed")
    return out


def sample_bands(p, tables, T, kind, u_b, u_g, ref_wall_edge=False):
    """Band and g point of emission for given uniforms, and the CDF rows
    searched: (nb, g, cdf_f, cdf_s, probq, row)."""
    T = np.ascontiguousarray(T, dtype=np.float32)
    ub = np.ascontiguousarray(u_b, np.float32)
    ug = np.ascontiguousarray(u_g, np.float32)
    n = ub.size
    nb = np.zeros(n, np.int32)
    g = np.zeros(n, np.int32)
    nB = 1000 if p.grey else p.nB
    nQ = 1 if p.grey else p.nQ
    cf, cs, pq = np.zeros(max(nB, p.grey_nB), np.float32), np.zeros(max(nB, p.grey_nB), np.float32), np.zeros(
        max(nQ, 1), np.float32)
    row = C.c_int()
    f = lib().oracle_sample_bands
    f.restype = C.c_int
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    f.argtypes = [C.POINTER(L.RcParams), C.POINTER(L.RcTables), C.POINTER(C.c_float), C.c_int, C.c_int,
                  C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_int),
                  C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int)]
    lib().oracle_set_ref_wall_edge(1 if ref_wall_edge else 0)
    try:
        rc = f(_pp(p), _tv(tables), _fp(T), kind, n, _fp(ub), _fp(ug), ip(nb), ip(g), _fp(cf), _fp(cs), _fp(pq),
               C.byref(row))
    finally:
        lib().oracle_set_ref_wall_edge(0)
    if rc != 0:
        raise RuntimeError("oracle_sample_bands failed: %d" % rc)
    nb_used = p.grey_nB if p.grey else p.nB
    return nb, g, cf[:nb_used], cs[:nb_used], pq[:nQ], row.value
