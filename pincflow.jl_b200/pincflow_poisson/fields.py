"""Caller-side state construction for the Poisson solve (host, numpy, FP64).

These functions build the inputs the reference's `State` holds when it
calls `solve_poisson!`: the terrain-following grid metric, the atmospheric
background and the sponge coefficient.  They restate, vectorised:

  Constants      src/Types/FoundationalTypes/Constants.jl:113-155
  Grid           src/Types/FoundationalTypes/Grid.jl:173-338
  topography     src/Types/FoundationalTypes/compute_topography.jl:145-176
  Atmosphere     src/Types/FoundationalTypes/Atmosphere.jl:278-323
  compute_n2!    src/Types/FoundationalTypes/compute_n2!.jl:43-82
  sponge         src/Update/compute_sponges!.jl:26-65

Array layout: numpy C order (k, j, i), which is the reference's
column-major (i, j, k) memory layout.  Haloed arrays have shape
(nz + 2 nbz, ny + 2 nby, nx + 2 nbx).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def constants() -> dict:
    gamma = 1.4
    kappa = (gamma - 1.0) / gamma
    rsp = 287.0
    g = 9.81
    rhoref = 1.184
    pref = 101325.0
    aref = math.sqrt(pref / rhoref)
    uref = aref
    lref = pref / rhoref / g
    tref = lref / aref
    thetaref = aref ** 2 / rsp
    g_ndim = g / (uref ** 2 / lref)
    ma = uref / aref
    fr = uref / math.sqrt(g * lref)
    sig = ma ** 2 / fr ** 2
    return dict(gamma=gamma, kappa=kappa, rsp=rsp, g=g, rhoref=rhoref, pref=pref, lref=lref,
                tref=tref, thetaref=thetaref, g_ndim=g_ndim, ma=ma, sig=sig)


@dataclass
class Domain:
    nx: int
    ny: int
    nz: int
    nbx: int = 3
    nby: int = 3
    nbz: int = 3

    @property
    def halo_shape(self):
        return (self.nz + 2 * self.nbz, self.ny + 2 * self.nby, self.nx + 2 * self.nbx)

    @property
    def interior_shape(self):
        return (self.nz, self.ny, self.nx)

    def interior(self, a):
        return a[self.nbz:self.nbz + self.nz, self.nby:self.nby + self.ny, self.nbx:self.nbx + self.nx]


def cell_centres(dom: Domain, lx: float, ly: float):
    """Dimensional interior cell centres x[i], y[j] (Grid.jl:199-210)."""
    xs = -lx / 2 + (np.arange(dom.nx) + 0.5) * (lx / dom.nx)
    ys = -ly / 2 + (np.arange(dom.ny) + 0.5) * (ly / dom.ny)
    return xs, ys


def _periodic_xy(dom: Domain, f: np.ndarray):
    """Periodic x and y halo fill (set_zonal/meridional_boundaries_of_field!).
    Modular indexing also covers nx < nbx or ny < nby (e.g. y_size = 1),
    where the reference's layer-by-layer copy repeats the interior."""
    bx, by = dom.nbx, dom.nby
    ix = bx + (np.arange(f.shape[-1]) - bx) % dom.nx
    iy = by + (np.arange(f.shape[-2]) - by) % dom.ny
    f[...] = f[..., ix]
    f[...] = f[..., iy, :]


def grid(dom: Domain, lx: float, ly: float, lz: float, hb_dim: np.ndarray,
         stretch_exp: float = 1.0) -> dict:
    """Terrain-following, vertically stretched grid (Grid.jl:173-338).

    lx, ly, lz dimensional [m]; hb_dim dimensional topography at the
    interior cell centres, shape (ny, nx); the stretching is
    z~(z^) = lz (z^/lz)^stretch_exp (identity for 1.0, the reference default).
    """
    c = constants()
    lref = c["lref"]
    nbx, nby, nbz = dom.nbx, dom.nby, dom.nbz
    lxn, lyn, lzn = lx / lref, ly / lref, lz / lref
    dx, dy, dz = lxn / dom.nx, lyn / dom.ny, lzn / dom.nz
    nzt = dom.nz + 2 * nbz
    z = (np.arange(nzt) - nbz) * dz + dz / 2

    def stretch(zh):
        return zh if stretch_exp == 1.0 else lz * (zh / lz) ** stretch_exp

    zt = np.empty(nzt)
    for k in range(nzt):
        level = z[k] + 0.5 * dz
        if level < 0:
            zt[k] = -stretch(-level * lref) / lref
        elif level > lzn:
            zt[k] = 2 * lzn - stretch((2 * lzn - level) * lref) / lref
        else:
            zt[k] = stretch(level * lref) / lref
    if np.any(np.diff(zt[nbz:nbz + dom.nz]) <= 0):
        raise ValueError("Error in Grid: Impossible vertical grid stretching!")
    zs = np.empty(nzt)
    zs[1:] = 0.5 * (zt[1:] + zt[:-1])
    zs[0] = zt[0] - 0.5 * (zt[2 * nbz - 1] - zt[2 * nbz - 2])

    nyy, nxx = dom.ny + 2 * nby, dom.nx + 2 * nbx
    hb = np.zeros((nyy, nxx))
    hb[nby:nby + dom.ny, nbx:nbx + dom.nx] = np.asarray(hb_dim, dtype=np.float64).reshape(dom.ny, dom.nx) / lref
    _periodic_xy(dom, hb)

    hs = dom.halo_shape
    jac = np.zeros(hs)
    m13 = np.zeros(hs)
    m23 = np.zeros(hs)
    m33 = np.zeros(hs)
    dzt = (zt[1:] - zt[:-1])[:, None, None]          # levels 1..nzz-1
    jac[1:] = (lzn - hb)[None] / lzn * dzt / dz
    jac[0] = jac[2 * nbz - 1]

    hx = np.zeros_like(hb)
    hy = np.zeros_like(hb)
    hx[:, 1:-1] = (hb[:, 2:] - hb[:, :-2]) / (2.0 * dx)
    hy[1:-1, :] = (hb[2:, :] - hb[:-2, :]) / (2.0 * dy)
    fac = (zs[1:, None, None] - lzn) / (lzn - hb)[None] * dz / dzt
    m13[1:] = hx[None] * fac
    m23[1:] = hy[None] * fac
    _periodic_xy(dom, m13)
    _periodic_xy(dom, m23)
    m13[0] = m13[2 * nbz - 1] * (zs[0] - lzn) / (zs[2 * nbz - 1] - lzn)
    m23[0] = m23[2 * nbz - 1] * (zs[0] - lzn) / (zs[2 * nbz - 1] - lzn)
    a2 = (lzn / (lzn - hb)) ** 2
    g2 = hx ** 2 + hy ** 2
    b = (zs[1:, None, None] - lzn) / (lzn - hb)[None]
    m33[1:] = (a2[None] + b ** 2 * g2[None]) * (dz / dzt) ** 2
    b0 = (zs[0] - lzn) / (lzn - hb)
    m33[0] = (a2 + b0 ** 2 * g2) * (dz / (zt[2 * nbz - 1] - zt[2 * nbz - 2])) ** 2
    _periodic_xy(dom, m33)
    zc = (lzn - hb)[None] / lzn * zs[:, None, None] + hb[None]
    return dict(dx=dx, dy=dy, dz=dz, jac=jac, met13=m13, met23=m23, met33=m33, zc=zc, hb=hb)


def atmosphere_stable(dom: Domain, buoyancy_frequency=1e-2, potential_temperature=300.0) -> dict:
    """Boussinesq, StableStratification (Atmosphere.jl:278-296)."""
    c = constants()
    hs = dom.halo_shape
    rhobar = np.ones(hs)
    thetabar = potential_temperature / c["thetaref"] * np.ones(hs)
    pbar = rhobar * thetabar
    n2 = (buoyancy_frequency * c["tref"]) ** 2 * np.ones(hs)
    return dict(pbar=pbar, thetabar=thetabar, rhobar=rhobar, n2=n2)


def atmosphere_isothermal(dom: Domain, g: dict, temperature=300.0, ground_pressure=1e5) -> dict:
    """Isothermal background (Atmosphere.jl:298-323) with compute_n2!.jl:57-79."""
    c = constants()
    t0 = temperature / c["thetaref"]
    p0 = ground_pressure / c["pref"]
    zc = g["zc"]
    pbar = p0 * np.exp(-c["sig"] * zc / c["gamma"] / t0)
    thetabar = t0 * np.exp(c["kappa"] * c["sig"] / t0 * zc)
    rhobar = pbar / thetabar
    n2 = np.zeros_like(pbar)
    k0, k1 = dom.nbz, dom.nbz + dom.nz - 1
    jac, dz = g["jac"], g["dz"]
    n2[k0:k1 + 1] = (c["g_ndim"] / thetabar[k0:k1 + 1] / jac[k0:k1 + 1] * 0.5
                     * (thetabar[k0 + 1:k1 + 2] - thetabar[k0 - 1:k1]) / dz)
    bot = c["g_ndim"] / thetabar[k0 - 1] / jac[k0 - 1] * (thetabar[k0] - thetabar[k0 - 1]) / dz
    top = c["g_ndim"] / thetabar[k1 + 1] / jac[k1 + 1] * (thetabar[k1 + 1] - thetabar[k1]) / dz
    for l in range(1, dom.nbz + 1):
        n2[k0 - l] = bot
        n2[k1 + l] = top
    return dict(pbar=pbar, thetabar=thetabar, rhobar=rhobar, n2=n2)


def sponge_sin2(dom: Domain, g: dict, zr: float, lz: float, dt: float) -> np.ndarray:
    """RHS sponge of the periodic-hill example (compute_sponges!.jl:38-64 with
    src/Examples/periodic_hill.jl:36-37): sin^2(pi/2 (z - zr)/(lz - zr)) / dt above zr."""
    c = constants()
    betar = np.zeros(dom.halo_shape)
    zcdim = dom.interior(g["zc"]) * c["lref"]
    dtdim = dt * c["tref"]
    val = np.where(zcdim >= zr, np.sin(np.pi / 2 * (zcdim - zr) / (lz - zr)) ** 2 / dtdim, 0.0)
    dom.interior(betar)[...] = val * c["tref"]
    _periodic_xy(dom, betar)
    k0, k1 = dom.nbz, dom.nbz + dom.nz - 1
    betar[k0 - 1] = betar[k0]
    betar[k1 + 1] = betar[k1]
    return betar


def fcscal(dom: Domain, f: dict) -> np.ndarray:
    """sqrt(pbar^2 / rhobar) on the interior (compute_operator!.jl:85)."""
    pb = dom.interior(f["pbar"])
    return np.sqrt(pb ** 2 / dom.interior(f["rhobar"]))


def consistent_projection(dom: Domain, f: dict, b: np.ndarray) -> np.ndarray:
    """Removes from b its component along the operator's left null vector
    w = J * fcscal (periodic x, y and solid walls make the scaled operator
    singular; a divergence right-hand side from compute_lhs! satisfies
    sum(w * b) = 0).  Returns b - (w.b / w.w) w."""
    w = dom.interior(f["jac"]) * fcscal(dom, f)
    return b - (np.vdot(w, b) / np.vdot(w, w)) * w
