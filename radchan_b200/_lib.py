"""ctypes declarations of the C ABI in include/radchan.h.

The shared library is built in-tree (radchan_b200/libradchan.so); importing
this module fails loudly when it is missing -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# RADCHAN_LIB=checked loads the bounds-checked build (libradchan_checked.so)
LIB_PATH = os.path.join(HERE, "libradchan_checked.so" if os.environ.get("RADCHAN_LIB") == "checked"
                        else "libradchan.so")

RC_MAX_LEVELS = 9
RC_OK = 0
RC_E = {-1: "RC_E_INVALID", -2: "RC_E_CUDA", -3: "RC_E_NOMEM", -4: "RC_E_IO", -5: "RC_E_STATE",
        -6: "RC_E_RANGE", -7: "RC_E_BUSY", -8: "RC_E_NOTFOUND", -9: "RC_E_CANCELLED",
        -10: "RC_E_TIMEOUT"}
RC_WEST, RC_EAST, RC_SOUTH, RC_NORTH, RC_BOT, RC_TOP = range(6)


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
_DP = C.POINTER(C.c_double)


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
                ("ksca", _FP), ("kabs", _FP), ("theta", _FP), ("phase_cdf", _FP)]


class RcScatterSpec(C.Structure):
    _fields_ = [("nB", C.c_int), ("nQ", C.c_int), ("nA", C.c_int),
                ("ksca_lo", C.c_double), ("ksca_hi", C.c_double),
                ("g_lo", C.c_double), ("g_hi", C.c_double),
                ("seed", C.c_uint64)]


class RcBundleId(C.Structure):
    _fields_ = [("kind", C.c_int), ("i", C.c_int), ("j", C.c_int), ("k", C.c_int), ("v", C.c_int),
                ("h", C.c_int)]


class RcTraceRec(C.Structure):
    _fields_ = [("nb", C.c_int), ("g", C.c_int), ("nsteps", C.c_int), ("end_level", C.c_int),
                ("sx", C.c_float), ("sy", C.c_float), ("sz", C.c_float), ("tra", C.c_float),
                ("De", C.c_double)]


class RcSolveInfo(C.Structure):
    _fields_ = [("Tmax", C.c_float), ("kappamax", C.c_float), ("Ibmax_fluid", C.c_float),
                ("table_row", C.c_int), ("status", C.c_int), ("bundles", C.c_double),
                ("steps", C.c_double), ("ms_device", C.c_float), ("ms_solve", C.c_float)]


class RcRequest(C.Structure):
    _fields_ = [("params", C.POINTER(RcParams)), ("table_set", C.c_int), ("T", _FP), ("zstart", C.c_int),
                ("tolerance", C.c_float)]


class RcResultInfo(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("photmax", C.c_int), ("rel_std_maxq", C.c_float), ("status", C.c_int)]


RC_DNS_MAX_T = 128


class RcDnsCoupling(C.Structure):
    _fields_ = [("Tin", C.c_double), ("Height", C.c_double), ("underrelax", C.c_double), ("stefan", C.c_double),
                ("nTemp", C.c_int), ("Tnb", C.POINTER(C.c_double)), ("kP", C.POINTER(C.c_double)),
                ("jstart", C.c_int), ("jend", C.c_int)]


# (name, restype, argtypes) for every function declared in include/radchan.h
_VP = C.c_void_p
_I = C.c_int
_SIGS = [
    ("rc_params_default", _I, [C.POINTER(RcParams)]),
    ("rc_params_from_headers", _I, [C.c_char_p, C.c_char_p, C.POINTER(RcParams)]),
    ("rc_params_validate", _I, [C.POINTER(RcParams), C.c_char_p, C.c_size_t]),
    ("rc_tables_synthetic", _I, [C.POINTER(RcSynthSpec), C.POINTER(_VP)]),
    ("rc_tables_read_dir", _I, [C.c_char_p, _I, _I, _I, C.POINTER(_VP)]),
    ("rc_tables_write_dir", _I, [_VP, C.c_char_p]),
    ("rc_tables_view", _I, [_VP, C.POINTER(RcTables)]),
    ("rc_tables_validate", _I, [C.POINTER(RcTables), C.c_char_p, C.c_size_t]),
    ("rc_tables_free", None, [_VP]),
    ("rc_scattering_synthetic", _I, [C.POINTER(RcScatterSpec), C.POINTER(_VP)]),
    ("rc_scattering_read_dir", _I, [C.c_char_p, _I, _I, C.POINTER(_VP)]),
    ("rc_scattering_write_dir", _I, [_VP, C.c_char_p]),
    ("rc_scattering_validate", _I, [C.POINTER(RcScattering), C.c_char_p, C.c_size_t]),
    ("rc_scattering_view", _I, [_VP, C.POINTER(RcScattering)]),
    ("rc_scattering_free", None, [_VP]),
    ("rc_create", _I, [C.POINTER(RcParams), _I, C.POINTER(_VP)]),
    ("rc_set_tables", _I, [_VP, C.POINTER(RcTables)]),
    ("rc_set_scattering", _I, [_VP, C.POINTER(RcScattering)]),
    ("rc_solve_async", _I, [_VP, _FP, _I, C.POINTER(C.c_int32)]),
    ("rc_solve_device_async", _I, [_VP, _VP, _I, C.POINTER(C.c_int32)]),
    ("rc_collect", _I, [_VP, C.c_int32, _FP, _FP, _DP, _DP, _DP, _DP]),
    ("rc_collect_device", _I, [_VP, C.c_int32, _VP, _VP, _VP, _VP]),
    ("rc_device_results", _I, [_VP, C.c_int32, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP)]),
    ("rc_solve_info_get", _I, [_VP, C.c_int32, C.POINTER(RcSolveInfo)]),
    ("rc_set_launch", _I, [_VP, _I, _I, _I, _I]),
    ("rc_set_priority", _I, [_VP, C.c_float]),
    ("rc_get_launch", _I, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("rc_autotune", _I, [_VP, _FP, _I, _I, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                         C.POINTER(C.c_int)]),
    ("rc_solve_noalloc", _I, [_VP, _VP, _I, _VP, _VP, _VP, _VP]),
    ("rc_destroy", _I, [_VP]),
    ("rc_get_params", _I, [_VP, C.POINTER(RcParams), C.POINTER(C.c_int)]),
    ("rc_slab_range", _I, [_I, _I, _I, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("rc_slab_unique_id", _I, [C.c_char_p]),
    ("rc_slab_comm_create", _I, [_I, _I, _I, C.c_char_p, C.c_double, C.POINTER(_VP)]),
    ("rc_slab_solve", _I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("rc_slab_last_error", _I, [_VP, C.c_char_p, C.c_size_t]),
    ("rc_slab_comm_destroy", _I, [_VP]),
    ("rc_last_error", _I, [_VP, C.c_char_p, C.c_size_t]),
    ("rc_debug_fail_next", _I, [C.c_char_p, _I]),
    ("rc_grid_level", _I, [C.POINTER(RcParams), _I, _FP, _FP, _FP, _FP, _FP, _FP]),
    ("rc_trace", _I, [_VP, C.c_int32, _I, C.POINTER(RcBundleId), C.POINTER(RcTraceRec), _I, C.POINTER(C.c_int)]),
    ("rc_probe_gather", _I, [_I, C.c_size_t, _I, _I, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    ("rc_sample_bands", _I, [_VP, C.c_int32, _I, _I, _FP, _FP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("rc_batch_create", _I, [_I, _I, C.POINTER(_VP)]),
    ("rc_batch_add", _I, [_VP, _VP, _FP, _I]),
    ("rc_batch_run", _I, [_VP]),
    ("rc_batch_wait", _I, [_VP, C.POINTER(C.c_float)]),
    ("rc_batch_phases", _I, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    ("rc_batch_collect", _I, [_VP, _I, _FP, _FP, _DP, _DP, _DP, _DP]),
    ("rc_batch_destroy", _I, [_VP]),
    ("rc_server_create", _I, [_I, C.c_double, _I, C.POINTER(_VP)]),
    ("rc_server_add_tables", _I, [_VP, C.POINTER(RcTables), C.POINTER(C.c_int)]),
    ("rc_server_set_scattering", _I, [_VP, _I, C.POINTER(RcScattering)]),
    ("rc_server_submit", _I, [_VP, C.POINTER(RcRequest), C.POINTER(C.c_int64)]),
    ("rc_server_wait", _I, [_VP, C.c_int64, _FP, _FP, C.POINTER(RcResultInfo)]),
    ("rc_server_stats", _I, [_VP, _DP, _DP, _DP]),
    ("rc_server_destroy", _I, [_VP]),
    ("rc_server_set_quantum", _I, [_VP, C.c_longlong]),
    ("rc_server_quanta", _I, [_VP, C.POINTER(C.c_longlong)]),
    ("rc_server_set_policy", _I, [_VP, _I]),
    ("rc_server_cancel", _I, [_VP, C.c_int64]),
    ("rc_dns_source", _I, [_VP, C.c_int32, C.POINTER(RcDnsCoupling), _DP, _DP, _DP, _DP, _DP,
                           C.POINTER(C.c_longlong)]),
    ("rc_dns_source_device", _I, [_VP, C.c_int32, C.POINTER(RcDnsCoupling), _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("rc_legacy_source", _I, [C.POINTER(RcDnsCoupling), _DP, _DP, _DP, _DP, _DP, C.POINTER(C.c_longlong)]),
    ("rc_legacy_configure", _I, [C.POINTER(RcParams), C.POINTER(RcTables)]),
    ("rc_legacy_release", _I, []),
    ("mc_gpu_", None, [_FP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("get_results_", None, [_FP, _FP, C.POINTER(C.c_int)]),
]

SYMBOLS = [s[0] for s in _SIGS]

_lib = None


def lib():
    """The loaded libradchan.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("radchan_b200/libradchan.so is missing: run python -m radchan_b200.build "
                               "(or __graft_entry__.build()) first")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error(ctx=None) -> str:
    buf = C.create_string_buffer(1024)
    lib().rc_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


class RadChanError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (RC_E.get(code, str(code)), msg))
        self.code = code


def check(rc, ctx=None):
    if rc != RC_OK:
        raise RadChanError(rc, last_error(ctx))
    return rc


def check_slab(rc, comm=None):
    """check() for the rc_slab_* calls (messages kept per communicator)."""
    if rc != RC_OK:
        buf = C.create_string_buffer(1024)
        lib().rc_slab_last_error(comm, buf, 1024)
        raise RadChanError(rc, buf.value.decode(errors="replace"))
    return rc
