"""Batched solves of ensemble members over the C ABI (pcf_ensemble_*).

The reference runs ensemble members as separate MPI sub-communicators
(src/ensemble.jl:40-43), each calling solve_poisson! on its own state.  Here
the members are PoissonSolver handles on one GPU, possibly of different grid
sizes; Ensemble.solve_poisson_device runs solve_poisson! for all of them
with the mixed-precision iteration, every batch of iterations of all members
being one CUDA graph launch.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .solver import PoissonNamelist, PoissonSolver, SolveInfo, _info


def _bind(lib):
    if getattr(lib, "_ens_bound", False):
        return lib
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    lib.pcf_ensemble_create.argtypes = [P(vp), P(vp), ctypes.c_int]
    lib.pcf_ensemble_destroy.argtypes = [vp]
    lib.pcf_ensemble_solve_device.argtypes = [vp, P(vp), P(vp), P(vp), P(vp), P(ctypes.c_double),
                                              P(ctypes.c_double), P(ctypes.c_double), P(_lib.PcfParams), P(vp),
                                              P(_lib.PcfResult)]
    lib.pcf_ensemble_launch_count.argtypes = [vp]
    lib.pcf_ensemble_launch_count.restype = ctypes.c_longlong
    for name in ("pcf_ensemble_create", "pcf_ensemble_destroy", "pcf_ensemble_solve_device"):
        getattr(lib, name).restype = ctypes.c_int
    lib._ens_bound = True
    return lib


class Ensemble:
    """Members advanced together; the solvers stay owned by the caller and
    must outlive the ensemble."""

    def __init__(self, solvers: list[PoissonSolver]):
        self.lib = _bind(_lib.load())
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        self._h = ctypes.c_void_p()
        _lib.check(self.lib.pcf_ensemble_create(ctypes.byref(self._h), arr, len(self.solvers)), "pcf_ensemble_create")

    def close(self):
        if self._h:
            self.lib.pcf_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launch_count(self) -> int:
        return int(self.lib.pcf_ensemble_launch_count(self._h))

    def solve_poisson_device(self, d_rhs, d_rho, d_betar, dt, rayleigh_factor, tolref, namelist: PoissonNamelist,
                             d_dpip, d_p=None) -> list[SolveInfo]:
        """solve_poisson! for every member: per-member raw device pointers
        (rhs interior, rho / betar / p / dpip haloed) and scalars."""
        n = len(self.solvers)
        vp = ctypes.c_void_p

        def ptrs(xs):
            return (vp * n)(*[vp(int(x)) if x else vp() for x in xs])

        def dbl(xs):
            return (ctypes.c_double * n)(*[float(x) for x in xs])

        res = (_lib.PcfResult * n)()
        prm = namelist.to_c()
        _lib.check(self.lib.pcf_ensemble_solve_device(self._h, ptrs(d_rhs), ptrs(d_rho), ptrs(d_betar),
                                                      ptrs(d_p) if d_p is not None else None, dbl(dt),
                                                      dbl(rayleigh_factor), dbl(tolref), ctypes.byref(prm),
                                                      ptrs(d_dpip), res), "pcf_ensemble_solve_device")
        return [_info(r) for r in res]
