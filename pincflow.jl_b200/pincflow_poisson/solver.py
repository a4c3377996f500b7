"""Host mirror of the reference's PoissonSolver interface over the C ABI.

Names and argument meanings follow the Julia functions they stand in for:

  PoissonNamelist          src/Types/NamelistTypes/PoissonNamelist.jl:38-66
  PoissonSolver.solve_poisson       solve_poisson!(state, dt, rayleigh_factor, tolref)
                                    src/PoissonSolver/solve_poisson!.jl:39-75
  PoissonSolver.compute_operator    compute_operator!(state, dt, rayleigh_factor)
  PoissonSolver.apply_operator      apply_operator!(sin, ls, Total()/Horizontal(), state)
  PoissonSolver.apply_preconditioner apply_preconditioner!(sin, sout, state)
  PoissonSolver.apply_bicgstab      apply_bicgstab!(state, tolref)
  PoissonSolver.compute_global_dot_product
                                    src/MPIOperations/compute_global_dot_product.jl:22-36

Error behaviour follows the reference: dt == 0 raises (solve_poisson!.jl:52-54);
non-convergence is returned as (errflag=True, niter) and leaves dpip
untouched (apply_bicgstab!.jl:146-149, solve_poisson!.jl:61-63).
Every compute call goes through libpincflow_poisson.so on the GPU; there
is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from .fields import Domain


@dataclass
class PoissonNamelist:
    tolerance: float = 1.0e-8
    poisson_iterations: int = 1000
    preconditioner: bool = True
    dtau: float = 1.0
    preconditioner_iterations: int = 2
    initial_cleaning: bool = True
    tolerance_is_relative: bool = False
    # SpongeNamelist.damp_horizontal_wind_on_rhs
    damp_horizontal_wind_on_rhs: bool = False
    # additions without a reference counterpart (defaults reproduce the reference)
    precision: str = "fp64"          # "fp64" | "mixed"
    residual: str = "recursive"      # "recursive" | "true"
    inner_tolerance: float = 1.0e-2   # mixed: residual drop between FP64 reliable updates
    max_refinements: int = 5          # mixed: restarts of the FP32 iteration after a breakdown
    learned: int = 0                  # mixed, bit set: 1 learned warm start, 2 learned preconditioner stage
    check_interval: int = 4
    restart_interval: int = 1         # mixed: Krylov restart at every n-th reliable update (0: never)
    multigrid: bool = False           # mixed: horizontal aggregation multigrid V-cycle as the preconditioner
    mg_dtau: float = 2.5              # multigrid: pseudo-time step of the smoother on every level
    mg_coarse_iterations: int = 4     # multigrid: smoothing steps on the coarsest level
    mg_min_columns: int = 16          # multigrid: a level with at most this many columns is the coarsest
    autotune: bool = False            # time the stencil tile shapes of each new grid size on first use
    mg_operator_bf16: bool = True     # multigrid: finest and first coarse level stencils read BF16 copies
    mg_fused_coarse: Optional[bool] = None  # multigrid: levels of <= 1024 columns as one cluster launch per cycle
    #                                         (None: in ensembles only)
    mg_smoother_fp8: bool = False     # multigrid: finest level's pseudo-time steps read an FP8 copy of their planes

    def to_c(self) -> _lib.PcfParams:
        p = _lib.PcfParams()
        _lib.load().pcf_params_default(ctypes.byref(p))
        p.tolerance = float(self.tolerance)
        p.poisson_iterations = int(self.poisson_iterations)
        p.preconditioner = int(bool(self.preconditioner))
        p.dtau = float(self.dtau)
        p.preconditioner_iterations = int(self.preconditioner_iterations)
        p.tolerance_is_relative = int(bool(self.tolerance_is_relative))
        p.damp_horizontal_wind_on_rhs = int(bool(self.damp_horizontal_wind_on_rhs))
        p.precision = _lib.PRECISION[self.precision]
        p.residual = _lib.RESIDUAL[self.residual]
        p.inner_tolerance = float(self.inner_tolerance)
        p.max_refinements = int(self.max_refinements)
        p.learned = int(self.learned)
        p.check_interval = int(self.check_interval)
        p.restart_interval = int(self.restart_interval)
        p.multigrid = int(bool(self.multigrid))
        p.mg_dtau = float(self.mg_dtau)
        p.mg_coarse_iterations = int(self.mg_coarse_iterations)
        p.mg_min_columns = int(self.mg_min_columns)
        p.autotune = int(bool(self.autotune))
        p.mg_operator_bf16 = int(bool(self.mg_operator_bf16))
        p.mg_fused_coarse = -1 if self.mg_fused_coarse is None else int(bool(self.mg_fused_coarse))
        p.mg_smoother_fp8 = int(bool(self.mg_smoother_fp8))
        return p


@dataclass
class SolveInfo:
    errflag: bool
    niter: int
    nrefine: int = 0
    status: int = 0
    residual: float = 0.0
    true_residual: float = 0.0
    b_norm: float = 0.0
    timings_ms: dict = field(default_factory=dict)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class PoissonSolver:
    """One device-resident solver instance: the `Poisson` workspace of one
    `State` (src/Types/PoissonTypes/Poisson.jl:53-89) plus the grid and
    background fields the operator is assembled from."""

    def __init__(self, dom: Domain, model: str = "PseudoIncompressible", device: int = 0):
        self.lib = _lib.load()
        self.dom = dom
        self.model = model
        d = _lib.PcfDims(dom.nx, dom.ny, dom.nz, dom.nbx, dom.nby, dom.nbz, _lib.MODEL[model], device)
        self._h = ctypes.c_void_p()
        _lib.check(self.lib.pcf_create(ctypes.byref(self._h), ctypes.byref(d)), "pcf_create")

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._h:
            self.lib.pcf_destroy(self._h)
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
    def device_bytes(self) -> int:
        return int(self.lib.pcf_device_bytes(self._h))

    @property
    def launch_count(self) -> int:
        return int(self.lib.pcf_launch_count(self._h))

    def profile(self, on: bool = True):
        _lib.check(self.lib.pcf_profile_enable(self._h, int(bool(on))), "pcf_profile_enable")

    def attach_network(self, net):
        """Use a trained LearnedNet as the warm start of mixed-precision solves
        with PoissonNamelist(learned=True); None detaches."""
        from .learned import attach
        attach(self, net)

    def test_stall_staged_copy(self, level: int, wait_limit_s: float = 1e-3):
        """Test hook of the failure path: the TMA-staged stencils skip the copy
        of z-level `level` and bound every copy wait by wait_limit_s, so that
        the next solve gives up with status PCF_ECUDA; level < 0 turns it off."""
        _lib.check(self.lib.pcf_test_stall_staged_copy(self._h, int(level), float(wait_limit_s)),
                   "pcf_test_stall_staged_copy")

    def residual_history(self) -> np.ndarray:
        """Relative recursive residual after each iteration of the last solve."""
        n = ctypes.c_int()
        _lib.check(self.lib.pcf_residual_history(self._h, None, 0, ctypes.byref(n)), "pcf_residual_history")
        out = np.zeros(max(n.value, 1))
        _lib.check(self.lib.pcf_residual_history(self._h, _lib.dptr(out), n.value, ctypes.byref(n)),
                   "pcf_residual_history")
        return out[:n.value]

    def profile_read(self) -> dict:
        out = {}
        for tag, name in enumerate(_lib.PROF_TAGS):
            ms, cnt, by = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
            _lib.check(self.lib.pcf_profile_read(self._h, tag, ctypes.byref(ms), ctypes.byref(cnt),
                                                 ctypes.byref(by)), "pcf_profile_read")
            out[name] = dict(ms=ms.value, count=cnt.value, bytes=by.value)
        return out

    # -- state ------------------------------------------------------------
    def set_grid(self, g: dict):
        self._keep_grid = [_f64(g[k]) for k in ("jac", "met13", "met23", "met33")]
        _lib.check(self.lib.pcf_set_grid(self._h, g["dx"], g["dy"], g["dz"],
                                         *[_lib.dptr(a) for a in self._keep_grid]), "pcf_set_grid")
        self.dx, self.dy, self.dz = g["dx"], g["dy"], g["dz"]

    def set_background(self, a: dict):
        th = _f64(a["thetabar"]) if a.get("thetabar") is not None else None
        arrs = [_f64(a["pbar"]), _f64(a["rhobar"]), th, _f64(a["n2"])]
        _lib.check(self.lib.pcf_set_background(self._h, *[_lib.dptr(x) for x in arrs]),
                   "pcf_set_background")

    # -- the reference's entry points ------------------------------------
    def solve_poisson(self, rhs, rho, betar, dt, rayleigh_factor, tolref, namelist: PoissonNamelist,
                      dpip, p=None) -> SolveInfo:
        """solve_poisson!: returns SolveInfo (errflag, niter, ...) and writes
        the interior of the haloed array dpip in place."""
        if dt == 0.0:
            raise ZeroDivisionError("Error in solve_poisson!: dt = 0.0!")
        if not (isinstance(dpip, np.ndarray) and dpip.dtype == np.float64 and dpip.flags["C_CONTIGUOUS"]):
            raise TypeError("dpip must be a C-contiguous float64 array")
        res = _lib.PcfResult()
        prm = namelist.to_c()
        args = [_f64(rhs), _f64(rho), _f64(betar), None if p is None else _f64(p)]
        _lib.check(self.lib.pcf_solve(self._h, *[_lib.dptr(a) for a in args], float(dt),
                                      float(rayleigh_factor), float(tolref), ctypes.byref(prm),
                                      _lib.dptr(dpip), ctypes.byref(res)), "pcf_solve")
        return _info(res)

    def compute_lhs(self, u, v, w, heating=None):
        """compute_lhs!: (rhs, tolref) from the haloed staggered winds (mass
        fluxes in the Compressible model, with the heating field)."""
        rhs = np.zeros(self.dom.interior_shape)
        tol = ctypes.c_double()
        h = None if heating is None else _f64(heating)
        _lib.check(self.lib.pcf_compute_lhs(self._h, _lib.dptr(_f64(u)), _lib.dptr(_f64(v)), _lib.dptr(_f64(w)),
                                            _lib.dptr(h), _lib.dptr(rhs), ctypes.byref(tol)), "pcf_compute_lhs")
        return rhs, tol.value

    def compute_lhs_device(self, d_u: int, d_v: int, d_w: int, d_rhs: int, d_heating: int | None = None) -> float:
        """compute_lhs! on device arrays (raw pointers); returns tolref."""
        tol = ctypes.c_double()
        _lib.check(self.lib.pcf_compute_lhs_device(self._h, ctypes.c_void_p(d_u), ctypes.c_void_p(d_v),
                                                   ctypes.c_void_p(d_w),
                                                   None if d_heating is None else ctypes.c_void_p(d_heating),
                                                   ctypes.c_void_p(d_rhs), ctypes.byref(tol)),
                   "pcf_compute_lhs_device")
        return tol.value

    def correct(self, dt, rayleigh_factor, dpip, u, v, w, rhop, pip, damp_horizontal_wind_on_rhs=False):
        """The corrector after solve_poisson (apply_corrector!.jl:58-61): fills
        dpip's halo and corrects u, v, w, rhop, pip, all haloed float64 arrays
        modified in place (rho, betar, p of the last solve)."""
        arrs = [dpip, u, v, w, rhop, pip]
        for a in arrs:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]):
                raise TypeError("correct: arrays must be C-contiguous float64")
        _lib.check(self.lib.pcf_correct(self._h, float(dt), float(rayleigh_factor),
                                        int(bool(damp_horizontal_wind_on_rhs)), *[_lib.dptr(a) for a in arrs]),
                   "pcf_correct")

    def correct_device(self, dt, rayleigh_factor, d_dpip, d_u, d_v, d_w, d_rhop, d_pip,
                       damp_horizontal_wind_on_rhs=False):
        """correct on device arrays (raw pointers), in place."""
        ptrs = [ctypes.c_void_p(x) for x in (d_dpip, d_u, d_v, d_w, d_rhop, d_pip)]
        _lib.check(self.lib.pcf_correct_device(self._h, float(dt), float(rayleigh_factor),
                                               int(bool(damp_horizontal_wind_on_rhs)), *ptrs), "pcf_correct_device")

    def apply_corrector_device(self, d_u, d_v, d_w, d_rho, d_rhop, d_betar, d_pip, dt, rayleigh_factor,
                               namelist: PoissonNamelist, d_dpip, d_p=None, d_heating=None) -> SolveInfo:
        """apply_corrector!(state, dt, rayleigh_factor) on device arrays:
        compute_lhs!, solve_poisson!, dpip halos, correct!.  Returns the solve's
        SolveInfo; the fields stay uncorrected when info.errflag is set."""
        res = _lib.PcfResult()
        prm = namelist.to_c()
        vp = ctypes.c_void_p
        opt = lambda x: None if x is None else vp(x)  # noqa: E731
        _lib.check(self.lib.pcf_apply_corrector_device(self._h, vp(d_u), vp(d_v), vp(d_w), vp(d_rho), vp(d_rhop),
                                                       vp(d_betar), opt(d_p), vp(d_pip), opt(d_heating), float(dt),
                                                       float(rayleigh_factor), ctypes.byref(prm), vp(d_dpip),
                                                       ctypes.byref(res)), "pcf_apply_corrector_device")
        return _info(res)

    # ------------------------------------------------ implicit half step --

    def set_predictand_boundaries_device(self, d_rho, d_rhop, d_u, d_v, d_w, d_pip, d_p=None):
        """set_boundaries!(state, BoundaryPredictands()) on device arrays (raw
        pointers of haloed float64 fields), in place."""
        vp = ctypes.c_void_p
        opt = lambda x: None if x is None else vp(x)  # noqa: E731
        _lib.check(self.lib.pcf_set_predictand_boundaries_device(self._h, opt(d_rho), vp(d_rhop), vp(d_u), vp(d_v),
                                                                 vp(d_w), vp(d_pip), opt(d_p)),
                   "pcf_set_predictand_boundaries_device")

    def modify_compressible_wind_device(self, d_p, d_u, d_v, d_w, divide=False):
        """modify_compressible_wind!(state, * or /) on device arrays, in place."""
        vp = ctypes.c_void_p
        _lib.check(self.lib.pcf_modify_compressible_wind_device(self._h, None if d_p is None else vp(d_p), vp(d_u),
                                                                vp(d_v), vp(d_w), int(bool(divide))),
                   "pcf_modify_compressible_wind_device")

    def implicit_predictor_device(self, dt, rayleigh_factor, d_u, d_v, d_w, d_rho, d_rhop, d_pip, d_betar, d_p=None,
                                  d_dudt=None, d_dvdt=None, d_wold=None, damp_horizontal_wind_on_rhs=False):
        """implicit_integration!.jl:53-63 on device arrays: wold = w, the
        implicit U, V, W updates, set_boundaries!, the implicit RhoP update,
        set_boundaries!.  d_dudt/d_dvdt: WKB tendencies or None (NoWKB)."""
        vp = ctypes.c_void_p
        opt = lambda x: None if x is None else vp(x)  # noqa: E731
        _lib.check(self.lib.pcf_implicit_predictor_device(
            self._h, float(dt), float(rayleigh_factor), int(bool(damp_horizontal_wind_on_rhs)), vp(d_u), vp(d_v),
            vp(d_w), vp(d_rho), vp(d_rhop), vp(d_pip), opt(d_p), vp(d_betar), opt(d_dudt), opt(d_dvdt), opt(d_wold)),
            "pcf_implicit_predictor_device")

    def implicit_step_device(self, dt, rayleigh_factor, namelist: PoissonNamelist, d_u, d_v, d_w, d_rho, d_rhop,
                             d_pip, d_betar, d_dpip, d_p=None, d_dudt=None, d_dvdt=None, d_heating=None,
                             d_wold=None) -> SolveInfo:
        """implicit_integration!.jl:49-77 without output on device arrays:
        the predictor, apply_corrector! and the compressible wind factors.
        Returns the solve's SolveInfo; on info.errflag the fields are the
        predicted, uncorrected ones."""
        res = _lib.PcfResult()
        prm = namelist.to_c()
        vp = ctypes.c_void_p
        opt = lambda x: None if x is None else vp(x)  # noqa: E731
        _lib.check(self.lib.pcf_implicit_step_device(
            self._h, float(dt), float(rayleigh_factor), ctypes.byref(prm), vp(d_u), vp(d_v), vp(d_w), vp(d_rho),
            vp(d_rhop), vp(d_pip), opt(d_p), vp(d_betar), opt(d_dudt), opt(d_dvdt), opt(d_heating), opt(d_wold),
            vp(d_dpip), ctypes.byref(res)), "pcf_implicit_step_device")
        return _info(res)

    def implicit_step(self, dt, rayleigh_factor, namelist: PoissonNamelist, u, v, w, rho, rhop, pip, betar, dpip,
                      p=None, dudt=None, dvdt=None, heating=None, wold=None) -> SolveInfo:
        """implicit_step_device with host arrays: u, v, w, rho, rhop, pip, p,
        dpip (and wold, if given) are C-contiguous float64 arrays updated in
        place; heating is interior, the rest haloed."""
        for a in (u, v, w, rho, rhop, pip, dpip, p, wold):
            if a is not None and not (isinstance(a, np.ndarray) and a.dtype == np.float64
                                      and a.flags["C_CONTIGUOUS"]):
                raise TypeError("implicit_step: in-place arrays must be C-contiguous float64")
        betar, dudt, dvdt, heating = (None if a is None else _f64(a) for a in (betar, dudt, dvdt, heating))
        res = _lib.PcfResult()
        prm = namelist.to_c()
        args = [u, v, w, rho, rhop, pip, p, betar, dudt, dvdt, heating, wold, dpip]
        _lib.check(self.lib.pcf_implicit_step(self._h, float(dt), float(rayleigh_factor), ctypes.byref(prm),
                                              *[_lib.dptr(a) for a in args], ctypes.byref(res)),
                   "pcf_implicit_step")
        return _info(res)

    def compute_operator(self, rho, betar, dt, rayleigh_factor, damp_horizontal_wind_on_rhs=False,
                         p=None, return_coef=True):
        coef = np.zeros((_lib.NCOEF,) + self.dom.interior_shape) if return_coef else None
        args = [_f64(rho), _f64(betar), None if p is None else _f64(p)]
        _lib.check(self.lib.pcf_compute_operator(self._h, *[_lib.dptr(a) for a in args], float(dt),
                                                 float(rayleigh_factor),
                                                 int(bool(damp_horizontal_wind_on_rhs)),
                                                 _lib.dptr(coef)), "pcf_compute_operator")
        return coef

    def set_operator(self, coef):
        c = _f64(coef)
        _lib.check(self.lib.pcf_set_operator(self._h, _lib.dptr(c)), "pcf_set_operator")

    def apply_operator(self, sin, horizontal=False, precision="fp64"):
        out = np.zeros(self.dom.interior_shape)
        _lib.check(self.lib.pcf_apply_operator(self._h, _lib.dptr(_f64(sin)), _lib.dptr(out),
                                               _lib.HORIZONTAL if horizontal else _lib.TOTAL,
                                               _lib.PRECISION[precision]), "pcf_apply_operator")
        return out

    def apply_preconditioner(self, sin, namelist: PoissonNamelist, precision="fp64"):
        out = np.zeros(self.dom.interior_shape)
        prm = namelist.to_c()
        _lib.check(self.lib.pcf_apply_preconditioner(self._h, _lib.dptr(_f64(sin)), _lib.dptr(out),
                                                     ctypes.byref(prm), _lib.PRECISION[precision]),
                   "pcf_apply_preconditioner")
        return out

    def multigrid_levels(self, namelist: PoissonNamelist) -> list:
        """(nx, ny, nz) of every level of the multigrid hierarchy built for
        the current operator (finest first)."""
        prm = namelist.to_c()
        n = ctypes.c_int()
        dims = (ctypes.c_int * 96)()
        _lib.check(self.lib.pcf_multigrid_levels(self._h, ctypes.byref(prm), 32, ctypes.byref(n), dims),
                   "pcf_multigrid_levels")
        return [(dims[3 * q], dims[3 * q + 1], dims[3 * q + 2]) for q in range(min(n.value, 32))]

    def multigrid_operator(self, level: int, shape) -> np.ndarray:
        """The 25 planes of a multigrid level, shape (25, nz, ny, nx)."""
        nx, ny, nz = shape
        out = np.zeros((_lib.NCOEF, nz, ny, nx))
        _lib.check(self.lib.pcf_multigrid_operator(self._h, int(level), _lib.dptr(out)), "pcf_multigrid_operator")
        return out

    def apply_multigrid(self, sin, namelist: PoissonNamelist):
        """One multigrid V-cycle z = MG(sin) (FP32 on the device)."""
        out = np.zeros(self.dom.interior_shape)
        prm = namelist.to_c()
        _lib.check(self.lib.pcf_apply_multigrid(self._h, _lib.dptr(_f64(sin)), _lib.dptr(out), ctypes.byref(prm)),
                   "pcf_apply_multigrid")
        return out

    def apply_bicgstab(self, rhs, tolref, namelist: PoissonNamelist):
        sol = np.zeros(self.dom.interior_shape)
        res = _lib.PcfResult()
        prm = namelist.to_c()
        _lib.check(self.lib.pcf_bicgstab(self._h, _lib.dptr(_f64(rhs)), float(tolref), ctypes.byref(prm),
                                         _lib.dptr(sol), ctypes.byref(res)), "pcf_bicgstab")
        return sol, _info(res)

    def compute_global_dot_product(self, a, b) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.pcf_global_dot(self._h, _lib.dptr(_f64(a)), _lib.dptr(_f64(b)),
                                           ctypes.byref(out)), "pcf_global_dot")
        return out.value

    def solve_poisson_device(self, d_rhs: int, d_rho: int, d_betar: int, dt, rayleigh_factor, tolref,
                             namelist: PoissonNamelist, d_dpip: int, d_p: int | None = None) -> SolveInfo:
        """solve_poisson! on device-resident inputs (raw device pointers)."""
        res = _lib.PcfResult()
        prm = namelist.to_c()
        _lib.check(self.lib.pcf_solve_device(self._h, ctypes.c_void_p(d_rhs), ctypes.c_void_p(d_rho),
                                             ctypes.c_void_p(d_betar),
                                             None if d_p is None else ctypes.c_void_p(d_p), float(dt),
                                             float(rayleigh_factor), float(tolref), ctypes.byref(prm),
                                             ctypes.c_void_p(d_dpip), ctypes.byref(res)),
                   "pcf_solve_device")
        return _info(res)


def autotune_entries() -> list:
    """The stencil tile choices the autotuner has made in this process."""
    lib = _lib.load()
    n = ctypes.c_int()
    _lib.check(lib.pcf_autotune_entries(None, 0, ctypes.byref(n)), "pcf_autotune_entries")
    arr = (_lib.PcfTuneEntry * max(n.value, 1))()
    _lib.check(lib.pcf_autotune_entries(arr, n.value, ctypes.byref(n)), "pcf_autotune_entries")
    out = []
    for e in arr[:n.value]:
        d = {name: getattr(e, name) for name, _ in e._fields_}
        d["kernel"] = _lib.TUNE_KERNELS[e.kernel]
        out.append(d)
    return out


def autotune_clear():
    _lib.check(_lib.load().pcf_autotune_clear(), "pcf_autotune_clear")


def _info(res: _lib.PcfResult) -> SolveInfo:
    d = res.as_dict()
    return SolveInfo(errflag=bool(d["errflag"]), niter=int(d["niter"]), nrefine=int(d["nrefine"]),
                     status=int(d["status"]), residual=d["residual"], true_residual=d["true_residual"],
                     b_norm=d["b_norm"],
                     timings_ms={k[3:]: d[k] for k in d if k.startswith("ms_")})
