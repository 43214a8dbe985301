"""radchan_b200 -- B200 (sm_100a) narrow-band correlated-k OERM Monte Carlo
radiative-transfer solver, a drop-in for RadChan's src/montecarlo GPU path.

The solver is libradchan.so (C++/CUDA behind include/radchan.h); this
package is its Python mirror (ctypes) plus the seeded synthetic workloads.
"""
from ._lib import RadChanError, lib  # noqa: F401
from .api import (Batch, Result, Solver, TableSet, copy_params, default_params, field_shape,  # noqa: F401
                  grid_level, params_from_headers, result_shape, set_levels, validate)
