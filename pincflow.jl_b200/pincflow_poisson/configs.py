"""Seeded synthetic workloads of the five benchmark configurations.

The reference publishes no benchmark inputs for its Poisson solve, so each
configuration is synthesised here with the shapes, sizes and value
distributions of its description:

  c1  periodic hill (src/Examples/periodic_hill.jl:13-37): Boussinesq, stable
      stratification, 40 x 1 x 40, lx = 20 km, ly = 1 km, lz = 20 km,
      h(x) = 250 (1 + cos(pi x / 10 km)) m, sin^2 RHS sponge above 10 km;
      the right-hand sides of the 200 solves of 100 time steps are seeded
      N(0,1) fields (consistent-projected) with rayleigh_factor alternating
      1.0 / 2.0 and dt = 1 s.
  c2  256 x 256 x 128 pseudo-incompressible, lx = ly = 100 km, lz = 20 km,
      stretched grid z~ = lz (z^/lz)^1.5, Gaussian mountain
      h = 1 km exp(-r^2 / (10 km)^2), isothermal 250 K, RHS N(0,1) seed 12345.
  c3  training set: 128 x 128 x 64 (lx = ly = 100 km, lz = 20 km), terrain a
      sum of 1-5 Gaussian hills (height U(0, 1.5 km), width U(5, 20 km)),
      Boussinesq with N ~ U(0.005, 0.02) 1/s, RHS N(0,1); seed = solve index.
  c4  32 solves, nx = ny in {64, 96, 128, 192}, nz = nx/2, terrain and N as c3.
  c5  512 x 512 x 192 pseudo-incompressible, lx = ly = 400 km, lz = 40 km,
      20 seeded Gaussian ridges (h <= 2 km), isothermal 250 K, RHS a 3-D
      Gaussian-envelope wave packet (kx = kz = 2 pi / 10 km, amplitude 1e-3)
      plus N(0, 1e-2) noise.
All right-hand sides are made consistent with the singular operator by
projecting out the left null vector (fields.consistent_projection); dt = 1
(non-dimensional, the initial-cleaning convention) unless stated.
"""
from __future__ import annotations

import numpy as np

from . import fields as F


def _periodic_offset(x, c, L):
    return (x - c + L / 2) % L - L / 2


def gaussian_hills(xs, ys, lx, ly, rng, nhills, hmax, wmin, wmax, ridge=False):
    X, Y = np.meshgrid(xs, ys)
    h = np.zeros_like(X)
    for _ in range(nhills):
        xc, yc = rng.uniform(-lx / 2, lx / 2), rng.uniform(-ly / 2, ly / 2)
        amp = rng.uniform(0, hmax)
        w = rng.uniform(wmin, wmax)
        dx = _periodic_offset(X, xc, lx)
        dy = _periodic_offset(Y, yc, ly)
        if ridge:
            th = rng.uniform(0, np.pi)
            u = dx * np.cos(th) + dy * np.sin(th)
            v = -dx * np.sin(th) + dy * np.cos(th)
            h += amp * np.exp(-(u / w) ** 2 - (v / (4 * w)) ** 2)
        else:
            h += amp * np.exp(-(dx ** 2 + dy ** 2) / w ** 2)
    return h


def _finish(dom, model, g, atm, rhs, dt, rf, betar=None, seed=0, name=""):
    f = dict(g)
    f.update(atm)
    rho = np.zeros(dom.halo_shape)
    if betar is None:
        betar = np.zeros(dom.halo_shape)
    rhs = F.consistent_projection(dom, f, rhs)
    return dict(name=name, dom=dom, model=model, fields=f, rho=rho, betar=betar, rhs=rhs, dt=dt,
                rayleigh_factor=rf, tolref=1.0, seed=seed)


def c1(seed: int = 0, step: int = 0):
    dom = F.Domain(40, 1, 40)
    lx, ly, lz = 20000.0, 1000.0, 20000.0
    xs, _ = F.cell_centres(dom, lx, ly)
    hb = (500.0 / 2 * (1 + np.cos(np.pi / 10000.0 * xs)))[None, :]
    g = F.grid(dom, lx, ly, lz, hb)
    atm = F.atmosphere_stable(dom, 1e-2, 300.0)
    c = F.constants()
    dt = 1.0 / c["tref"]
    betar = F.sponge_sin2(dom, g, 10000.0, lz, dt)
    rng = np.random.default_rng(1000 + seed * 1000 + step)
    rhs = rng.standard_normal(dom.interior_shape)
    rf = 1.0 if step % 2 == 0 else 2.0
    return _finish(dom, "Boussinesq", g, atm, rhs, dt, rf, betar, seed, "c1")


def c2(seed: int = 12345, nx: int = 256, ny: int = 256, nz: int = 128):
    dom = F.Domain(nx, ny, nz)
    lx, ly, lz = 100e3, 100e3, 20e3
    xs, ys = F.cell_centres(dom, lx, ly)
    X, Y = np.meshgrid(xs, ys)
    hb = 1000.0 * np.exp(-(X ** 2 + Y ** 2) / 10e3 ** 2)
    g = F.grid(dom, lx, ly, lz, hb, stretch_exp=1.5)
    atm = F.atmosphere_isothermal(dom, g, temperature=250.0)
    rng = np.random.default_rng(seed)
    rhs = rng.standard_normal(dom.interior_shape)
    return _finish(dom, "PseudoIncompressible", g, atm, rhs, 1.0, 1.0, None, seed, "c2")


def c3(index: int, nx: int = 128, ny: int = 128, nz: int = 64):
    dom = F.Domain(nx, ny, nz)
    lx, ly, lz = 100e3, 100e3, 20e3
    rng = np.random.default_rng(index)
    xs, ys = F.cell_centres(dom, lx, ly)
    hb = gaussian_hills(xs, ys, lx, ly, rng, int(rng.integers(1, 6)), 1500.0, 5e3, 20e3)
    g = F.grid(dom, lx, ly, lz, hb)
    atm = F.atmosphere_stable(dom, float(rng.uniform(0.005, 0.02)), 300.0)
    rhs = rng.standard_normal(dom.interior_shape)
    return _finish(dom, "Boussinesq", g, atm, rhs, 1.0, 1.0, None, index, "c3")


def c4_sizes(seed: int = 4, count: int = 32):
    rng = np.random.default_rng(seed)
    return [int(v) for v in rng.choice([64, 96, 128, 192], size=count)]


def c4(index: int, nx: int):
    return c3(10_000 + index, nx=nx, ny=nx, nz=nx // 2) | {"name": "c4"}


def c5(seed: int = 5, nx: int = 512, ny: int = 512, nz: int = 192, lx: float = 400e3, ly: float = 400e3,
       ridges: int = 20):
    """The large domain; smaller lx, ly and ridge counts give patches of the
    same family at the same resolution (training data of the learned part)."""
    dom = F.Domain(nx, ny, nz)
    lz = 40e3
    rng = np.random.default_rng(seed)
    xs, ys = F.cell_centres(dom, lx, ly)
    hb = gaussian_hills(xs, ys, lx, ly, rng, ridges, 2000.0, 5e3, 20e3, ridge=True)
    if hb.max() > 2000.0:
        hb *= 2000.0 / hb.max()
    g = F.grid(dom, lx, ly, lz, hb)
    atm = F.atmosphere_isothermal(dom, g, temperature=250.0)
    c = F.constants()
    zc = dom.interior(g["zc"]) * c["lref"]
    X = xs[None, None, :]
    Y = ys[None, :, None]
    k = 2 * np.pi / 10e3
    env = np.exp(-((X / 40e3) ** 2 + (Y / 40e3) ** 2 + ((zc - lz / 2) / (lz / 6)) ** 2))
    rhs = 1e-3 * env * np.cos(k * X + k * zc) + 1e-2 * rng.standard_normal(dom.interior_shape)
    return _finish(dom, "PseudoIncompressible", g, atm, rhs, 1.0, 1.0, None, seed, "c5")


def c5_patch(index: int, n: int = 128):
    """An n x n x 192 patch of the c5 family at c5's resolution (781 m x
    781 m cells, lz = 40 km), with ridges in proportion to its area and its own
    seed: the learned part's training problems for the c5 workload."""
    frac = n / 512
    return c5(seed=20_000 + index, nx=n, ny=n, nz=192, lx=400e3 * frac, ly=400e3 * frac,
              ridges=max(1, round(20 * frac * frac))) | {"name": "c5_patch"}


CONFIGS = {"c1": c1, "c2": c2, "c3": c3, "c5": c5}
