"""B200 (sm_100a) implementation of the INS2D explicit time-stepping hot path:
time_ERK over the energy-conserving staggered finite-volume right-hand side F
and the pressure-Poisson projection (PCG and FFT), behind the C-ABI of
include/ins2d.h (libins2d.so)."""
from .api import (F, Ensemble, Ins2dError, Options, check_conservation, pressure_additional_solve, pressure_poisson,
                  time_ERK)
from .rk import getRKmethod

__all__ = ["Options", "Ensemble", "Ins2dError", "F", "pressure_poisson", "pressure_additional_solve", "time_ERK",
           "check_conservation", "getRKmethod"]
