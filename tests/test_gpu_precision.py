"""Precision study: the FP32 march with its FP64 tally against the full-FP64
build of the same kernels with the same Philox streams, per cell and per
wall cell, in units of the Monte Carlo standard deviation.  Optically thick
tables, emissivity 0.8, specular y walls, adiabatic x walls with wall
fluxes, nVar 8 (the 192x128x128 study's physics at a size a test affords)."""
import numpy as np
import pytest

from radchan_b200 import api
from radchan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_fp32_march_within_a_small_fraction_of_sigma_of_fp64():
    tabs = W.tables_nb(logk_lo=-1.0, logk_hi=2.0)
    p32 = W.channel_params(48, 32, 32, photmax=128, nVar=8, bd_y=3, eps=0.8, adiabw=1, adiabe=1, calcwalls=1,
                           levels=[(48, 32, 32), (24, 16, 16)], maxs=[5, 100000])
    p64 = api.copy_params(p32)
    p64.floatpoint = 1
    T = W.channel_field(p32, seed=17)
    r32 = api.Solver(p32, tabs).solve(T)
    r64 = api.Solver(p64, tabs).solve(T)
    st = api.compare_in_sigma(r32, r64)
    # identical draws: the builds differ only by rounding, which is far below
    # the Monte Carlo noise (tolerance: rounding may flip a near-tie crossing
    # or a CDF boundary for a few bundles of a cell)
    assert st["cells"]["rms_z"] < 0.05, st
    assert st["cells"]["max_abs_z"] < 0.5, st
    assert abs(st["cells"]["mean_z"]) < 0.01, st
    assert st["walls"]["rms_z"] < 0.05, st
    assert st["walls"]["max_abs_z"] < 0.5, st
