"""B200 (sm_100a) FP64 time-step engine for the LittleHarsh channel DNS.

Host-side mirror of the reference's Fortran surface over the C ABI in
include/lh_gpu.h: :class:`Engine` is one channel instance (start, the RK3
substep, LUsolU/LUsolP, four_to_phys/phys_to_four), :class:`Batch` advances
many instances in shared launches, :mod:`lh_b200.serve` runs the request
loop, :mod:`lh_b200.state` builds initial conditions and reads/writes the
reference's spectral files.
"""
from .capi import (DT_CFL, DT_FIXED, GRID_POLY, GRID_TANH, Batch, Desc, Engine, LHError,  # noqa: F401
                   host_grid, lib)
from .state import grids, perturbed_laminar, re_from_retau, read_state, write_state  # noqa: F401
