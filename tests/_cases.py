"""Small seeded cases shared by the oracle and GPU parity tests."""
from __future__ import annotations

import numpy as np

from pincflow_poisson import configs as C
from pincflow_poisson import fields as F


def _perturb(cfg, seed, rho_amp=0.0, betar_amp=0.0, compressible=False):
    dom = cfg["dom"]
    rng = np.random.default_rng(seed)
    if rho_amp:
        rho = rho_amp * rng.standard_normal(dom.halo_shape) * cfg["fields"]["rhobar"]
        cfg["rho"] = np.ascontiguousarray(rho)
    if betar_amp:
        cfg["betar"] = np.ascontiguousarray(betar_amp * rng.random(dom.halo_shape))
    if compressible:
        cfg["model"] = "Compressible"
        cfg["p"] = np.ascontiguousarray(cfg["fields"]["pbar"] * (1 + 0.01 * rng.standard_normal(dom.halo_shape)))
    return cfg


def case(name: str):
    """Returns a config dict (see configs._finish) plus optional 'p', 'damp'."""
    if name == "hill":          # periodic hill, y_size = 1, sponge
        cfg = C.c1(seed=0, step=1)
    elif name == "mtn":         # stretched terrain-following PI grid
        cfg = C.c2(nx=48, ny=40, nz=24)
    elif name == "odd":         # odd sizes: scalar paths and partial tiles
        cfg = C.c3(7, nx=37, ny=29, nz=13)
    elif name == "rho":         # density fluctuation, Rayleigh damping on all faces
        cfg = _perturb(C.c2(nx=32, ny=16, nz=12, seed=3), 11, rho_amp=0.05, betar_amp=0.3)
        cfg["damp"] = True
        cfg["rayleigh_factor"] = 2.0
        cfg["dt"] = 0.7
    elif name == "comp":        # compressible model (dpdpi term, thetabar buoyancy factor)
        cfg = _perturb(C.c2(nx=24, ny=20, nz=10, seed=4), 12, rho_amp=0.02, betar_amp=0.1, compressible=True)
        cfg["dt"] = 0.5
    elif name == "wide":        # wide tile path (nx >= 128)
        cfg = C.c3(9, nx=160, ny=12, nz=20)
    elif name == "oddx":        # odd nx, even ny: multigrid aggregates 1 x 2 columns
        cfg = C.c3(5, nx=25, ny=32, nz=12)
    elif name == "wide2":       # wide tile with partial x and y tiles (136 = 128 + 8, 10 = 2 x 4 + 2)
        cfg = C.c3(13, nx=136, ny=10, nz=12)
    elif name == "wide3":       # 512 wide: the V-cycle's staged stencils take 64-wide tiles; partial y tile
        cfg = C.c3(15, nx=512, ny=10, nz=8)
    else:
        raise KeyError(name)
    cfg.setdefault("damp", False)
    cfg.setdefault("p", None)
    return cfg


CASES = ["hill", "mtn", "odd", "rho", "comp", "wide"]


def oracle_operator(O, cfg):
    dom = cfg["dom"]
    d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    f = cfg["fields"]
    return d, O.compute_operator(d, O.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                                 cfg["rayleigh_factor"], cfg["damp"], cfg["p"])


def consistent_rhs(O, cfg):
    """A right-hand side in the range of the operator.  With rho' = 0 the
    operator's left null vector is J * fcscal and the configs' projected
    N(0,1) fields are consistent.  With rho' != 0 the horizontally varying
    buoyancy factor breaks that identity (at the 1e-5 level for these random
    fields), so the right-hand side is manufactured as b = A x* instead."""
    if not np.any(cfg["rho"]):
        return cfg["rhs"]
    d, coef = oracle_operator(O, cfg)
    x = np.random.default_rng(cfg["seed"] + 99).standard_normal(cfg["dom"].interior_shape)
    return O.apply_operator(d, coef, x)


def iterations_agree(a, b):
    """BiCGSTAB iteration counts at 1e-10 move by several iterations under
    1e-16 input perturbations (measured on the oracle: 73..80 for one case),
    so parity allows max(8, 15 %)."""
    return abs(a - b) <= max(8, 0.15 * max(a, b))


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def null_weights(cfg):
    dom = cfg["dom"]
    f = cfg["fields"]
    return dom.interior(f["jac"]) * F.fcscal(dom, f)
