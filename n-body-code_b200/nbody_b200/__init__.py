"""nbody_b200 - Python binding of the B200 Hermite-4 N-body engine.

The compute path is libnbody_cuda.so (hand-written sm_100a kernels behind the
C-ABI in include/nbody_cuda.h); this package only marshals arguments.
"""
from ._lib import LIB_PATH, NBodyError, header_functions, load
from .engine import (Engine, FIELDS, force_calculation, force_calculation_tune, measure_peaks, plummer, reference_ic,
                     release_force_cache)
from .adjoint import Adjoint, hermite_rollout
from .ensemble import Ensemble, plummer_ensemble

__all__ = [
    "Adjoint", "Engine", "Ensemble", "hermite_rollout", "plummer_ensemble", "FIELDS", "LIB_PATH", "NBodyError", "force_calculation", "force_calculation_tune", "header_functions", "load",
    "measure_peaks", "plummer", "reference_ic", "release_force_cache",
]
