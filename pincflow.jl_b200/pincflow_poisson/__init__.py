"""B200 (sm_100a) drop-in for PinCFlow.jl's semi-implicit pressure Poisson solve.

The compute lives in libpincflow_poisson.so (include/pincflow_poisson.h);
this package is its host-side mirror of the reference interface
(PoissonSolver.solve_poisson, apply_operator, apply_preconditioner, ...)
plus the caller-side construction of the grid, background and workloads.
"""
from . import configs, fields
from ._lib import PoissonError, load
from .ensemble import Ensemble
from .solver import PoissonNamelist, PoissonSolver, SolveInfo, autotune_clear, autotune_entries

__all__ = ["PoissonNamelist", "PoissonSolver", "SolveInfo", "PoissonError", "load", "fields", "configs",
           "autotune_entries", "autotune_clear", "Ensemble"]
