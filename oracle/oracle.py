"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is a literal FP64 C++ restatement of PinCFlow.jl's Poisson path
(see pcf_oracle.h for the per-function reference citations).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module;
the product never imports it.

Parity status: PARITY UNPINNED by reference golden vectors (the reference
ships none for the Poisson path and Julia cannot run here); pinned instead to
analytic known-answer tests in tests/test_oracle_kat.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpcf_oracle.so")

NCOEF = 25
# Plane order of the reference Tensor struct (src/Types/PoissonTypes/Tensor.jl:70-96).
COEF_NAMES = ["ac", "al", "ar", "ab", "af", "ad", "au", "ald", "alu", "ard", "aru", "abd",
              "abu", "afd", "afu", "add", "auu", "aldd", "aluu", "ardd", "aruu", "abdd",
              "abuu", "afdd", "afuu"]
MODELS = {"Boussinesq": 0, "PseudoIncompressible": 1, "Compressible": 2}


class Dims(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("nx", "ny", "nz", "nbx", "nby", "nbz", "ko", "z_size")]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        d = ctypes.POINTER(ctypes.c_double)
        _lib.or_dot.restype = ctypes.c_double
        _lib.or_compute_lhs.restype = ctypes.c_double
        _lib.or_compute_lhs_compressible.restype = ctypes.c_double
        _lib.or_grid.restype = ctypes.c_int
        _lib.or_solve_poisson.restype = ctypes.c_int
        del d
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _pn(a):
    return None if a is None else _p(a)


def dims(nx, ny, nz, nb=3):
    return Dims(nx, ny, nz, nb, nb, nb, 0, nz)


def halo_shape(d: Dims):
    """Shape of a haloed field in C order (k, j, i): x is fastest as in Julia."""
    return (d.nz + 2 * d.nbz, d.ny + 2 * d.nby, d.nx + 2 * d.nbx)


def interior_shape(d: Dims):
    return (d.nz, d.ny, d.nx)


def set_threads(n: int):
    lib().or_set_threads(int(n))


def get_threads() -> int:
    return lib().or_get_threads()


def constants() -> dict:
    out = np.zeros(12)
    lib().or_constants(_p(out))
    keys = ["gamma", "kappa", "rsp", "g", "rhoref", "pref", "lref", "tref", "thetaref",
            "g_ndim", "ma", "sig"]
    return dict(zip(keys, out.tolist()))


def grid(d: Dims, lx, ly, lz, stretch_exp, hb_dim):
    hs = halo_shape(d)
    jac, m13, m23, m33, zc = (np.zeros(hs) for _ in range(5))
    dxyz = np.zeros(3)
    hb = np.ascontiguousarray(hb_dim, dtype=np.float64).reshape(d.ny, d.nx)
    rc = lib().or_grid(ctypes.byref(d), ctypes.c_double(lx), ctypes.c_double(ly),
                       ctypes.c_double(lz), ctypes.c_double(stretch_exp), _p(hb), _p(jac),
                       _p(m13), _p(m23), _p(m33), _p(zc), _p(dxyz))
    if rc != 0:
        raise ValueError("impossible vertical grid stretching")
    return dict(jac=jac, met13=m13, met23=m23, met33=m33, zc=zc, dx=dxyz[0], dy=dxyz[1],
                dz=dxyz[2])


def atmosphere(d: Dims, background: int, params, jac, zc, dz):
    hs = halo_shape(d)
    pbar, thetabar, rhobar, n2 = (np.zeros(hs) for _ in range(4))
    prm = np.asarray(params, dtype=np.float64)
    rc = lib().or_atmosphere(ctypes.byref(d), background, _p(prm), _p(jac), _p(zc),
                             ctypes.c_double(dz), _p(pbar), _p(thetabar), _p(rhobar), _p(n2))
    assert rc == 0
    return dict(pbar=pbar, thetabar=thetabar, rhobar=rhobar, n2=n2)


def sponge_sin2(d: Dims, zc, zr, lz, dt):
    betar = np.zeros(halo_shape(d))
    lib().or_sponge_sin2(ctypes.byref(d), _p(zc), ctypes.c_double(zr), ctypes.c_double(lz),
                         ctypes.c_double(dt), _p(betar))
    return betar


def compute_operator(d: Dims, model, f: dict, rho, betar, dt, rayleigh_factor,
                     damp_horizontal_wind_on_rhs=False, p=None):
    coef = np.zeros((NCOEF,) + interior_shape(d))
    lib().or_compute_operator(
        ctypes.byref(d), int(model), ctypes.c_double(f["dx"]), ctypes.c_double(f["dy"]),
        ctypes.c_double(f["dz"]), _p(f["jac"]), _p(f["met13"]), _p(f["met23"]),
        _p(f["met33"]), _p(f["pbar"]), _p(f["rhobar"]), _pn(f.get("thetabar")), _p(f["n2"]),
        _p(rho), _p(betar), _pn(p), ctypes.c_double(dt), ctypes.c_double(rayleigh_factor),
        int(bool(damp_horizontal_wind_on_rhs)), _p(coef))
    return coef


def apply_operator(d: Dims, coef, s, horizontal=False):
    out = np.zeros(interior_shape(d))
    lib().or_apply_operator(ctypes.byref(d), _p(coef), _p(np.ascontiguousarray(s)), _p(out),
                            int(bool(horizontal)))
    return out


def apply_preconditioner(d: Dims, coef, dx, dy, dtau, iters, s):
    out = np.zeros(interior_shape(d))
    lib().or_apply_preconditioner(ctypes.byref(d), _p(coef), ctypes.c_double(dx),
                                  ctypes.c_double(dy), ctypes.c_double(dtau), int(iters),
                                  _p(np.ascontiguousarray(s)), _p(out))
    return out


def bicgstab(d: Dims, coef, dx, dy, rhs, tolerance=1e-8, poisson_iterations=1000,
             preconditioner=True, dtau=1.0, preconditioner_iterations=2,
             tolerance_is_relative=False, tolref=1.0):
    sol = np.zeros(interior_shape(d))
    out = np.zeros(4)
    lib().or_bicgstab(ctypes.byref(d), _p(coef), ctypes.c_double(dx), ctypes.c_double(dy),
                      ctypes.c_double(tolerance), int(poisson_iterations), int(bool(preconditioner)),
                      ctypes.c_double(dtau), int(preconditioner_iterations),
                      int(bool(tolerance_is_relative)), ctypes.c_double(tolref),
                      _p(np.ascontiguousarray(rhs)), _p(sol), _p(out))
    return sol, dict(errflag=bool(out[0]), niter=int(out[1]), residual=out[2], b_norm=out[3])


def solve_poisson(d: Dims, model, f: dict, rho, betar, rhs, dt, rayleigh_factor, tolref=1.0,
                  damp_horizontal_wind_on_rhs=False, p=None, tolerance=1e-8,
                  poisson_iterations=1000, preconditioner=True, dtau=1.0,
                  preconditioner_iterations=2, tolerance_is_relative=False):
    dpip = np.zeros(halo_shape(d))
    out = np.zeros(4)
    rc = lib().or_solve_poisson(
        ctypes.byref(d), int(model), ctypes.c_double(f["dx"]), ctypes.c_double(f["dy"]),
        ctypes.c_double(f["dz"]), _p(f["jac"]), _p(f["met13"]), _p(f["met23"]),
        _p(f["met33"]), _p(f["pbar"]), _p(f["rhobar"]), _pn(f.get("thetabar")), _p(f["n2"]),
        _p(rho), _p(betar), _pn(p), ctypes.c_double(dt), ctypes.c_double(rayleigh_factor),
        int(bool(damp_horizontal_wind_on_rhs)), ctypes.c_double(tolerance),
        int(poisson_iterations), int(bool(preconditioner)), ctypes.c_double(dtau),
        int(preconditioner_iterations), int(bool(tolerance_is_relative)),
        ctypes.c_double(tolref), _p(np.ascontiguousarray(rhs)), _p(dpip), _p(out))
    if rc != 0:
        raise ZeroDivisionError("Error in solve_poisson!: dt = 0.0!")
    return dpip, dict(errflag=bool(out[0]), niter=int(out[1]), residual=out[2], b_norm=out[3])


def compute_lhs(d: Dims, f: dict, u, v, w, model="PseudoIncompressible", heating=None):
    """compute_lhs!: (rhs, tolref); Compressible takes the heating field (interior, None: 0)."""
    c = constants()
    rhs = np.zeros(interior_shape(d))
    args = [ctypes.byref(d), ctypes.c_double(f["dx"]), ctypes.c_double(f["dy"]), ctypes.c_double(f["dz"]),
            ctypes.c_double(c["ma"]), ctypes.c_double(c["kappa"]), _p(f["jac"]), _p(f["pbar"]),
            _p(f["rhobar"]), _p(u), _p(v), _p(w)]
    if model == "Compressible":
        h = None if heating is None else np.ascontiguousarray(heating, dtype=np.float64)
        tolref = lib().or_compute_lhs_compressible(*args, _pn(h), _p(rhs))
    else:
        tolref = lib().or_compute_lhs(*args, _p(rhs))
    return rhs, tolref


def correct(d: Dims, model, f: dict, rho, betar, dt, rayleigh_factor, dpip, u, v, w, rhop, pip,
            damp_horizontal_wind_on_rhs=False, p=None):
    """apply_corrector!.jl:58-61 after the solve: fills dpip's halos and
    corrects u, v, w, rhop, pip; returns copies (dpip, u, v, w, rhop, pip)."""
    c = constants()
    out = [np.array(x, dtype=np.float64, copy=True) for x in (dpip, u, v, w, rhop, pip)]
    lib().or_correct(ctypes.byref(d), int(model), ctypes.c_double(f["dx"]), ctypes.c_double(f["dy"]),
                     ctypes.c_double(f["dz"]), _p(f["jac"]), _p(f["met13"]), _p(f["met23"]), _p(f["met33"]),
                     _p(f["rhobar"]), _p(f["pbar"]), _pn(f.get("thetabar")), _p(f["n2"]), _p(betar), _p(rho),
                     _pn(p), ctypes.c_double(dt), ctypes.c_double(rayleigh_factor),
                     int(bool(damp_horizontal_wind_on_rhs)), ctypes.c_double(1.0 / c["kappa"]),
                     ctypes.c_double(1.0 / c["ma"] ** 2), ctypes.c_double(c["g_ndim"]), *[_p(x) for x in out])
    return tuple(out)


def dot(a, b) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    b = np.ascontiguousarray(b, dtype=np.float64).ravel()
    return lib().or_dot(ctypes.c_long(a.size), _p(a), _p(b))


def set_predictand_boundaries(d: Dims, model, rho, rhop, u, v, w, pip, p=None):
    """set_boundaries!(state, BoundaryPredictands()) in place (model: int)."""
    pp = p if p is not None else np.zeros_like(rho)
    lib().or_set_predictand_boundaries(ctypes.byref(d), int(model), _p(rho), _p(rhop), _p(u), _p(v), _p(w),
                                       _p(pip), _p(pp))


def modify_compressible_wind(d: Dims, model, f: dict, p, u, v, w, divide=False):
    """modify_compressible_wind!(state, * or /) in place (Compressible only)."""
    if int(model) != 2:
        return
    lib().or_modify_compressible_wind(ctypes.byref(d), int(model), _p(f["jac"]), _p(p), _p(u), _p(v), _p(w),
                                      int(bool(divide)))


def implicit_predictor(d: Dims, model, f: dict, betar, dt, rayleigh_factor, rho, rhop, u, v, w, pip, p=None,
                       dudt=None, dvdt=None, damp_horizontal_wind_on_rhs=False):
    """implicit_integration!.jl:53-63 on copies: returns
    (rho, rhop, u, v, w, pip, p, wold) after save_backups!(:w), the implicit
    U, V, W updates, set_boundaries!, the implicit RhoP update and
    set_boundaries!.  model: int; dudt/dvdt None for NoWKB."""
    c = constants()
    out = [np.array(x, dtype=np.float64, copy=True) for x in (rho, rhop, u, v, w, pip)]
    pp = np.array(p if p is not None else np.zeros_like(rho), dtype=np.float64, copy=True)
    wold = np.zeros_like(out[4])
    lib().or_implicit_predictor(
        ctypes.byref(d), int(model), ctypes.c_double(f["dx"]), ctypes.c_double(f["dy"]), ctypes.c_double(f["dz"]),
        _p(f["jac"]), _p(f["met13"]), _p(f["met23"]), _p(f["met33"]), _p(f["rhobar"]), _p(f["pbar"]),
        _pn(f.get("thetabar")), _p(f["n2"]), _p(betar), _p(out[0]), _p(pp), ctypes.c_double(dt),
        ctypes.c_double(rayleigh_factor), int(bool(damp_horizontal_wind_on_rhs)), ctypes.c_double(1.0 / c["kappa"]),
        ctypes.c_double(1.0 / c["ma"] ** 2), ctypes.c_double(c["g_ndim"]), _pn(dudt), _pn(dvdt), _p(out[2]),
        _p(out[3]), _p(out[4]), _p(out[1]), _p(out[5]), _p(wold))
    return (*out, pp if p is not None else None, wold)


def implicit_step(d: Dims, model_name, f: dict, betar, dt, rayleigh_factor, rho, rhop, u, v, w, pip, p=None,
                  dudt=None, dvdt=None, heating=None, damp_horizontal_wind_on_rhs=False, **solver):
    """implicit_integration!.jl:49-77 without output, on copies:
    modify_compressible_wind!(*), set_boundaries!, the predictor (:53-63),
    apply_corrector! (compute_lhs!, solve_poisson!, dpip halos, correct!),
    modify_compressible_wind!(/), set_boundaries!.  Returns
    (fields dict, info); on errflag the fields are those after the
    predictor (the reference raises there)."""
    model = MODELS[model_name]
    rho, rhop, u, v, w, pip = [np.array(x, dtype=np.float64, copy=True) for x in (rho, rhop, u, v, w, pip)]
    p = None if p is None else np.array(p, dtype=np.float64, copy=True)
    modify_compressible_wind(d, model, f, p, u, v, w)
    set_predictand_boundaries(d, model, rho, rhop, u, v, w, pip, p)
    rho, rhop, u, v, w, pip, p, wold = implicit_predictor(
        d, model, f, betar, dt, rayleigh_factor, rho, rhop, u, v, w, pip, p=p, dudt=dudt, dvdt=dvdt,
        damp_horizontal_wind_on_rhs=damp_horizontal_wind_on_rhs)
    rhs, tolref = compute_lhs(d, f, u, v, w, model=model_name, heating=heating)
    dpip, info = solve_poisson(d, model, f, rho, betar, rhs, dt, rayleigh_factor, tolref=tolref,
                               damp_horizontal_wind_on_rhs=damp_horizontal_wind_on_rhs, p=p, **solver)
    out = dict(rho=rho, rhop=rhop, u=u, v=v, w=w, pip=pip, p=p, wold=wold, dpip=dpip, rhs=rhs)
    if info["errflag"]:
        return out, info
    dpip, u, v, w, rhop, pip = correct(d, model, f, rho, betar, dt, rayleigh_factor, dpip, u, v, w, rhop, pip,
                                       damp_horizontal_wind_on_rhs=damp_horizontal_wind_on_rhs, p=p)
    modify_compressible_wind(d, model, f, p, u, v, w, divide=True)
    set_predictand_boundaries(d, model, rho, rhop, u, v, w, pip, p)
    out.update(rho=rho, rhop=rhop, u=u, v=v, w=w, pip=pip, p=p, dpip=dpip)
    return out, info
