"""parallel_ds_b200: a B200-native FP64 dual simplex engine.

Drop-in for the solver path of veret-v/parallel_ds (load LP -> solve ->
status / objective / primal / dual) behind the C ABI in include/ds_api.h.
Every per-iteration step runs in hand-written sm_100a kernels
(libds_b200.so); this package holds the ctypes binding, the host-side mirror
of the reference's Problem / CudaDualSimplex interface and the LP generator.
"""
from ._lib import DsError, lib  # noqa: F401
from .solver import (BoundaryType, CudaDualSimplex, LPsolution, Matrix, Problem,  # noqa: F401
                     solve_lp)

__all__ = ["BoundaryType", "CudaDualSimplex", "LPsolution", "Matrix", "Problem", "solve_lp", "lib",
           "DsError"]
