"""Arithmetic primitives and the C ABI surface (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from radchan_b200 import _lib as L
from radchan_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _olib():
    from oracle import oracle as O
    lib = O.lib()
    lib.oracle_math_probe.restype = C.c_int
    lib.oracle_math_probe.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.oracle_philox.restype = C.c_int
    lib.oracle_philox.argtypes = [C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    return lib


def probe(which, x, y=None, width=1):
    lib = _olib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    inp = x if y is None else np.concatenate([x, np.asarray(y, np.float64)])
    out = np.zeros(len(x) * width)
    assert lib.oracle_math_probe(which, len(x), inp.ctypes.data_as(C.POINTER(C.c_double)),
                                 out.ctypes.data_as(C.POINTER(C.c_double))) == 0
    return out.reshape(len(x), width) if width > 1 else out


# Known-answer vectors of Philox4x32-10 published with Random123 (kat_vectors):
# counter, key -> output
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers(ctr, key, expect):
    lib = _olib()
    c = (C.c_uint * 4)(*ctr)
    k = (C.c_uint * 2)(*key)
    o = (C.c_uint * 4)()
    lib.oracle_philox(c, k, o)
    assert tuple(o) == expect


def test_expf_error_bound():
    x = np.linspace(-87.0, 88.0, 400001).astype(np.float32).astype(np.float64)
    got = probe(0, x)
    ref = np.exp(x)
    ulp = np.spacing(ref.astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(got - ref) / ulp) <= 2.0


def test_expm1f_small_args_relative():
    x = np.concatenate([-np.logspace(-8, 0, 20001), np.logspace(-8, -0.5, 2001)]).astype(np.float32).astype(float)
    got = probe(1, x)
    ref = np.expm1(x)
    assert np.max(np.abs(got - ref) / np.abs(ref)) < 5e-7


def test_exp_double():
    x = np.linspace(-700, 700, 100001)
    got = probe(2, x)
    assert np.max(np.abs(got - np.exp(x)) / np.exp(x)) < 4e-16
    x = np.concatenate([-np.logspace(-12, 0, 1001), np.logspace(-12, -0.4, 1001)])
    assert np.max(np.abs(probe(3, x) - np.expm1(x)) / np.abs(np.expm1(x))) < 6e-16


def test_sincos2pi():
    u = np.linspace(0, 1, 200001).astype(np.float32).astype(float)
    sc = probe(4, u, width=2)
    assert np.max(np.abs(sc[:, 0] - np.sin(2 * np.pi * u))) < 2e-7
    assert np.max(np.abs(sc[:, 1] - np.cos(2 * np.pi * u))) < 2e-7
    sc = probe(5, u, width=2)
    assert np.max(np.abs(sc[:, 0] - np.sin(2 * np.pi * u))) < 1e-15


def test_planck_identities():
    # integral of pi*I_b over wavenumber equals sigma T^4 (to quadrature accuracy)
    nu = np.linspace(1.0, 40000.0, 400000)
    for T in (300.0, 1000.0, 2000.0):
        ib = probe(6, np.full_like(nu, T), nu)
        integral = np.pi * np.trapezoid(ib, nu * 100.0)
        assert abs(integral / (5.670373e-08 * T ** 4) - 1) < 2e-4
    # cold wall (T = 0) emits nothing
    assert probe(6, np.array([0.0]), np.array([1000.0]))[0] == 0.0


def _header_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|const char \*)\s+\**(\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = L.lib()  # loads without a GPU
    declared = _header_functions(os.path.join(ROOT, "include", "radchan.h"))
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(L.SYMBOLS)


def test_default_params_match_reference_header():
    p = api.default_params()
    assert (p.imax, p.jmax, p.kmax) == (406, 576, 2304)
    assert p.grid_num == 9 and list(p.maxi)[:9] == [406, 406, 406, 406, 406, 14, 14, 14, 2]
    assert list(p.maxs)[:9] == [5] * 8 + [100000]
    assert (p.nT, p.nQ, p.nB) == (135, 16, 999)
    assert list(p.bd) == [2, 2, 1, 1, 4, 4]
    assert api.validate(p) == ""


def test_validate_rejects_bad_params():
    p = api.default_params()
    p.num_gpu = 4
    assert "num_gpu" in api.validate(p)
    p = api.default_params()
    p.maxi[1] = 405
    assert api.validate(p)
    p = api.default_params()
    p.bd[2] = 7
    assert api.validate(p)
    p = api.default_params()
    p.p_col = 5
    assert "p_col" in api.validate(p)


def test_create_without_gpu_reports_error():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("GPU present")
    p = api.default_params()
    with pytest.raises(L.RadChanError):
        api.Solver(p)


def test_fortran_module_binds_declared_symbols_and_mirrors_structs():
    """fortran/radchan_mod.f90 (no Fortran compiler here): every bind(C)
    name is a function the header declares and the library exports, and
    each bind(C) derived type lists as many components as the C struct it
    mirrors."""
    src = open(os.path.join(ROOT, "fortran", "radchan_mod.f90")).read()
    names = re.findall(r'bind\(C,\s*name="(\w+)"\)', src)
    declared = set(_header_functions(os.path.join(ROOT, "include", "radchan.h")))
    lib = L.lib()
    assert len(names) >= 15
    for n in names:
        assert n in declared, n
        assert hasattr(lib, n), n
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "radchan.h")).read(), flags=re.S)
    for tname in ("rc_params", "rc_tables", "rc_scattering", "rc_dns_coupling"):
        body = re.search(r"type, bind\(C\), public :: %s\n(.*?)end type %s" % (tname, tname), src, flags=re.S).group(1)
        f_fields = []
        for line in body.splitlines():
            line = line.split("!")[0]
            if "::" not in line:
                continue
            decl = line.split("::")[1]
            f_fields += [x.strip().split("(")[0] for x in re.split(r",(?![^()]*\))", decl) if x.strip()]
        cbody = re.search(r"typedef struct %s \{(.*?)\} %s;" % (tname, tname), hdr, flags=re.S).group(1)
        c_fields = []
        for stmt in cbody.split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            decl = re.sub(r"^(const\s+)?(unsigned\s+)?\w+\s*\**", "", stmt)
            c_fields += [re.sub(r"[\s\*]|\[.*?\]", "", x) for x in decl.split(",") if x.strip()]
        assert [f.lower() for f in f_fields] == [c.lower() for c in c_fields], (tname, f_fields, c_fields)
