"""ctypes mirrors of the structures of include/radchan.h that the oracle's C
entry points take (rc_params, rc_tables, rc_synth_spec, rc_bundle_id,
rc_trace_rec).

TEST INFRASTRUCTURE ONLY.  The oracle declares its own copies so that it
loads without the product package: bench.py's reference arm builds its
workload and runs the oracle with libradchan.so never loaded.  Instances of
the product package's structures (same layout) are converted byte for byte
by `params()` / `tables_view()`.
"""
from __future__ import annotations

import ctypes as C

RC_MAX_LEVELS = 9


class RcParams(C.Structure):
    _fields_ = [
        ("imax", C.c_int), ("jmax", C.c_int), ("kmax", C.c_int),
        ("Lx", C.c_float), ("Ly", C.c_float), ("Lz", C.c_float),
        ("fact_mesh", C.c_double),
        ("nVar", C.c_int), ("photmax", C.c_int),
        ("chanHeight", C.c_double),
        ("grid_num", C.c_int),
        ("maxi", C.c_int * RC_MAX_LEVELS), ("maxj", C.c_int * RC_MAX_LEVELS),
        ("maxk", C.c_int * RC_MAX_LEVELS), ("maxs", C.c_int * RC_MAX_LEVELS),
        ("num_gpu", C.c_int), ("p_col", C.c_int),
        ("num_streams", C.c_int), ("blockdim", C.c_int), ("nblocks", C.c_int),
        ("srt", C.c_int), ("grey", C.c_int), ("calcwalls", C.c_int), ("random", C.c_int),
        ("floatpoint", C.c_int),
        ("eps", C.c_float * 6), ("Tw", C.c_float * 6),
        ("adiabw", C.c_int), ("adiabe", C.c_int),
        ("stefan", C.c_double),
        ("toll", C.c_float), ("tollS", C.c_float),
        ("bd", C.c_int * 6),
        ("grey_nT", C.c_int), ("grey_nB", C.c_int),
        ("abscoeff", C.c_float), ("Tmins", C.c_float), ("wvmax", C.c_float),
        ("nT", C.c_int), ("nQ", C.c_int), ("nB", C.c_int),
        ("seed", C.c_uint64),
    ]


_FP = C.POINTER(C.c_float)


class RcTables(C.Structure):
    _fields_ = [("nT", C.c_int), ("nB", C.c_int), ("nQ", C.c_int),
                ("Tnb", _FP), ("kP", _FP), ("wvl", _FP), ("wvr", _FP), ("wvc", _FP),
                ("kavg", _FP), ("kq", _FP), ("prob", _FP), ("probg", _FP), ("wq", _FP)]


class RcSynthSpec(C.Structure):
    _fields_ = [("nB", C.c_int), ("nQ", C.c_int), ("nT", C.c_int),
                ("T_lo", C.c_double), ("T_hi", C.c_double),
                ("nu_lo", C.c_double), ("nu_hi", C.c_double),
                ("logk_lo", C.c_double), ("logk_hi", C.c_double),
                ("nexp", C.c_double), ("kexp", C.c_double),
                ("seed", C.c_uint64)]


class RcScattering(C.Structure):
    _fields_ = [("nB", C.c_int), ("nQ", C.c_int), ("nA", C.c_int),
                ("ksca", C.POINTER(C.c_float)), ("kabs", C.POINTER(C.c_float)),
                ("theta", C.POINTER(C.c_float)), ("phase_cdf", C.POINTER(C.c_float))]


class RcBundleId(C.Structure):
    _fields_ = [("kind", C.c_int), ("i", C.c_int), ("j", C.c_int), ("k", C.c_int), ("v", C.c_int),
                ("h", C.c_int)]


class RcTraceRec(C.Structure):
    _fields_ = [("nb", C.c_int), ("g", C.c_int), ("nsteps", C.c_int), ("end_level", C.c_int),
                ("sx", C.c_float), ("sy", C.c_float), ("sz", C.c_float), ("tra", C.c_float),
                ("De", C.c_double)]


def params(p) -> RcParams:
    """The oracle's RcParams for any structure with rc_params' layout."""
    if isinstance(p, RcParams):
        return p
    assert C.sizeof(p) == C.sizeof(RcParams), "rc_params layout mismatch"
    return RcParams.from_buffer_copy(p)


def tables_view(view) -> RcTables:
    """The oracle's RcTables for any structure with rc_tables' layout (the
    pointers are copied, so the arrays must outlive the call)."""
    if isinstance(view, RcTables):
        return view
    assert C.sizeof(view) == C.sizeof(RcTables), "rc_tables layout mismatch"
    return RcTables.from_buffer_copy(view)
