"""Seeded tiny cases whose oracle outputs are stored in small_cases.npz."""
import numpy as np

from pincflow_poisson import configs as C
from pincflow_poisson import fields as F

GOLDEN = ["tiny_terrain", "tiny_compressible"]


def golden_case(name):
    if name == "tiny_terrain":
        # stretched terrain-following PI grid with a Gaussian mountain
        cfg = C.c2(seed=31, nx=8, ny=6, nz=6)
    elif name == "tiny_compressible":
        # compressible model with rho', Rayleigh damping on all faces
        cfg = C.c3(32, nx=6, ny=4, nz=5)
        dom = cfg["dom"]
        g = {k: cfg["fields"][k] for k in ("dx", "dy", "dz", "jac", "met13", "met23", "met33", "zc")}
        atm = F.atmosphere_isothermal(dom, g, temperature=260.0)
        cfg["fields"].update(atm)
        rng = np.random.default_rng(33)
        cfg["model"] = "Compressible"
        cfg["rho"] = 0.02 * rng.standard_normal(dom.halo_shape) * atm["rhobar"]
        cfg["betar"] = 0.2 * rng.random(dom.halo_shape)
        cfg["p"] = atm["pbar"] * (1 + 0.01 * rng.standard_normal(dom.halo_shape))
        cfg["damp"] = True
        cfg["dt"] = 0.6
        cfg["rayleigh_factor"] = 2.0
    else:
        raise KeyError(name)
    cfg.setdefault("damp", False)
    cfg.setdefault("p", None)
    return cfg
