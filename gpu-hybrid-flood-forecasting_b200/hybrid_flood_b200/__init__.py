"""B200-native (sm_100a) 2-D shallow-water finite-volume step.

A drop-in for the hot path of arsanjeevk/gpu-hybrid-flood-forecasting: the
reference solver's ``finite_volume_step`` / ``compute_cfl_dt`` /
``rainfall_rate`` / ``run`` (``src/hybrid_flood/numpy_solver/shallow_water_2d.py``,
``src/hybrid_flood/jax_solver/numerics.py``), executed by hand-written CUDA
kernels in ``libswe_b200.so`` (C ABI: ``include/swe_b200.h``).

Importing the package does not load the native library; the first solver call
does, and raises if it has not been built (there is no CPU fallback).
"""

from .boundary import OPEN, REFLECTIVE, BoundaryConfig, all_open, all_reflective, apply_ghost_cells

__version__ = "0.1.0"

__all__ = [
    "OPEN", "REFLECTIVE", "BoundaryConfig", "all_open", "all_reflective", "apply_ghost_cells",
    "B200ShallowWaterSolver", "SWEState", "RunResult", "finite_volume_step", "compute_cfl_dt",
    "rainfall_rate", "ledger_error",
]


def __getattr__(name):
    if name in {"B200ShallowWaterSolver", "SWEState", "RunResult", "finite_volume_step",
                "compute_cfl_dt", "rainfall_rate", "ledger_error", "DeviceParams"}:
        from . import solver

        return getattr(solver, name)
    raise AttributeError(name)
