"""Known-answer tests of the oracle's implicit half step (or_predict.cpp):
the predictand boundaries (set_boundaries!.jl:46-60), the implicit
predictor (implicit_integration!.jl:53-63 with update!.jl's Implicit()
methods) and the whole step around apply_corrector!.

These pin the restatement without reference vectors: the boundary fill
against its definition written with numpy index arithmetic, the predictor on
flat terrain against the closed forms it reduces to (the pressure-gradient
step for u, v and the implicit-Euler buoyancy oscillator for w, rho'), and
the whole step against the projection it ends with."""
import numpy as np
import pytest

from _cases import case, rel_err
from pincflow_poisson import fields as F

G_NDIM_KEY = "g_ndim"


def _flat(nx=12, ny=10, nz=8):
    dom = F.Domain(nx, ny, nz)
    g = F.grid(dom, 30e3, 20e3, 10e3, np.zeros((ny, nx)))
    f = dict(g)
    f.update(F.atmosphere_stable(dom, 0.012, 300.0))
    return dom, f


def _random_state(dom, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(dom.halo_shape) for _ in range(5)]  # u, v, w, rhop, pip


def _numpy_fill(dom, a, sign, staggered=False):
    """The boundary rule as index arithmetic: every ghost value copies the
    interior value at the periodic (x, y) position, reflected in z."""
    nb, nz = dom.nbz, dom.nz
    out = a.copy()
    zz, yy, xx = np.meshgrid(np.arange(a.shape[0]), np.arange(a.shape[1]), np.arange(a.shape[2]), indexing="ij")
    si = (xx - dom.nbx) % dom.nx + dom.nbx
    sj = (yy - dom.nby) % dom.ny + dom.nby
    kk = zz - nb
    if staggered:
        src = np.where(kk < -1, -kk - 2, np.where(kk >= nz, 2 * (nz - 1) - kk, kk))
        val = a[src + nb, sj, si] * np.where((kk < -1) | (kk >= nz), sign, 1.0)
        val = np.where((kk == -1) | (kk == nz - 1), 0.0, val)
        out = val
    else:
        src = np.where(kk < 0, -kk - 1, np.where(kk >= nz, 2 * nz - 1 - kk, kk))
        out = a[src + nb, sj, si] * np.where((kk < 0) | (kk >= nz), sign, 1.0)
    return out


@pytest.mark.parametrize("model", [0, 1, 2])
def test_predictand_boundaries_follow_the_wall_rules(model, oracle):
    dom, _ = _flat(7, 5, 6)
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    rng = np.random.default_rng(model)
    rho, rhop, u, v, w, pip, p = (rng.standard_normal(dom.halo_shape) for _ in range(7))
    want = dict(rhop=_numpy_fill(dom, rhop, -1.0), u=_numpy_fill(dom, u, 1.0), v=_numpy_fill(dom, v, 1.0),
                w=_numpy_fill(dom, w, -1.0, staggered=True), pip=_numpy_fill(dom, pip, 1.0),
                rho=_numpy_fill(dom, rho, -1.0) if model >= 1 else rho.copy(),
                p=_numpy_fill(dom, p, 1.0) if model == 2 else p.copy())
    oracle.set_predictand_boundaries(d, model, rho, rhop, u, v, w, pip, p)
    for name, got in dict(rho=rho, rhop=rhop, u=u, v=v, w=w, pip=pip, p=p).items():
        np.testing.assert_array_equal(got, want[name], err_msg=name)


def test_predictor_with_zero_time_step_changes_no_interior_value(oracle):
    cfg = case("mtn")
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    u, v, w, rhop, pip = _random_state(dom, 5)
    model = oracle.MODELS[cfg["model"]]
    rho2, rhop2, u2, v2, w2, pip2, _, wold = oracle.implicit_predictor(
        d, model, f, cfg["betar"], 0.0, 1.0, cfg["rho"], rhop, u, v, w, pip)
    I = dom.interior  # noqa: E741
    np.testing.assert_array_equal(wold, w)
    np.testing.assert_array_equal(I(u2), I(u))
    np.testing.assert_array_equal(I(v2), I(v))
    # w on the top wall is the boundary's zero; below it w is unchanged
    np.testing.assert_array_equal(I(w2)[:-1], I(w)[:-1])
    assert not I(w2)[-1].any()
    assert rel_err(I(rhop2), I(rhop)) < 4e-16
    np.testing.assert_array_equal(I(pip2), I(pip))


def test_predictor_on_flat_terrain_is_the_implicit_buoyancy_oscillator(oracle):
    """With met13 = met23 = 0, no damping and no WKB forcing the implicit
    predictor reduces to u' = u - dt G_x, v' = v - dt G_y (G the Exner
    pressure gradient), and per column to backward Euler for dw/dt = b - G_z,
    db/dt = -N^2 w: w' = (w + dt (b_e - G_z)) / (1 + N_e^2 dt^2) with the
    old buoyancy b = -g rho' / rho_tot, then b' = (b - dt N^2 J (wbar -
    dt Gbar)) / (1 + N^2 dt^2) with the old w averaged to the cell."""
    dom, f = _flat()
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    c = oracle.constants()
    g = c[G_NDIM_KEY]
    kinv = 1.0 / c["kappa"] / c["ma"] ** 2
    dt = 0.37
    u, v, w, rhop, pip = _random_state(dom, 8)
    rhop *= 1e-3
    for a in (u, v, w, rhop, pip):
        F._periodic_xy(dom, a)
    rho = np.zeros(dom.halo_shape)
    betar = np.zeros(dom.halo_shape)
    z = dom.nbz
    w[z - 1] = 0.0
    w[z + dom.nz - 1] = 0.0
    _, rhop2, u2, v2, w2, _, _, _ = oracle.implicit_predictor(d, 0, f, betar, dt, 1.0, rho, rhop, u, v, w, pip)
    J, rb, pb, n2, m33 = f["jac"], f["rhobar"], f["pbar"], f["n2"], f["met33"]
    sl = lambda a, di=0, dj=0, dk=0: a[z + dk:z + dk + dom.nz, dom.nby + dj:dom.nby + dj + dom.ny,  # noqa: E731
                                       dom.nbx + di:dom.nbx + di + dom.nx]
    # u at i + 1/2 and v at j + 1/2
    gx = kinv * 0.5 * (sl(pb) + sl(pb, 1)) / (0.5 * (sl(rb) + sl(rb, 1))) * (sl(pip, 1) - sl(pip)) / f["dx"]
    gy = kinv * 0.5 * (sl(pb) + sl(pb, 0, 1)) / (0.5 * (sl(rb) + sl(rb, 0, 1))) * (sl(pip, 0, 1) - sl(pip)) / f["dy"]
    assert rel_err(sl(u2), sl(u) - dt * gx) < 1e-13
    assert rel_err(sl(v2), sl(v) - dt * gy) < 1e-13
    # w at k + 1/2 for the levels below the top wall
    Jc, Ju = sl(J), sl(J, 0, 0, 1)
    wt = lambda a, b_: (Ju * a + Jc * b_) / (Jc + Ju)  # noqa: E731
    # on flat terrain the horizontal pi' terms of the W gradient carry met13 = met23 = 0
    gz = kinv * wt(sl(pb), sl(pb, 0, 0, 1)) / wt(sl(rb), sl(rb, 0, 0, 1)) * wt(sl(m33), sl(m33, 0, 0, 1)) * (
        sl(pip, 0, 0, 1) - sl(pip)) / f["dz"]
    b = -g * rhop / rb
    b_e = -g * (Ju * sl(rhop) / sl(rb) / Jc + Jc * sl(rhop, 0, 0, 1) / sl(rb, 0, 0, 1) / Ju) / (Jc + Ju)
    n2e = wt(sl(n2), sl(n2, 0, 0, 1))
    w_want = (sl(w) - dt * gz + dt * b_e) / (1.0 + n2e * dt ** 2)
    assert rel_err(sl(w2)[:-1], w_want[:-1]) < 1e-12
    # rho' in the cells, with the wall gradients zero
    gz_c = gz.copy()
    gz_c[-1] = 0.0
    gz_below = np.concatenate([np.zeros_like(gz[:1]), gz_c[:-1]])
    gbar = 0.5 * (gz_below + gz_c)
    wbar = 0.5 * (sl(w) + sl(w, 0, 0, -1))
    b_new = (sl(b) - dt * sl(n2) * sl(J) * (wbar - dt * gbar)) / (1.0 + sl(n2) * dt ** 2)
    assert rel_err(sl(rhop2), -b_new * sl(rb) / g) < 1e-12


@pytest.mark.parametrize("name", ["mtn", "hill"])
def test_implicit_step_ends_divergence_free(name, oracle):
    """The step's last change to the winds is the corrector's projection
    (after the predictor has made them divergent), so compute_lhs! of the
    returned winds vanishes to the solver tolerance."""
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    u, v, w, rhop, pip = _random_state(dom, 21)
    rhop *= 1e-3
    out, info = oracle.implicit_step(d, cfg["model"], f, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["rho"],
                                     rhop, u, v, w, pip, damp_horizontal_wind_on_rhs=cfg["damp"], tolerance=1e-13,
                                     tolerance_is_relative=True, poisson_iterations=5000)
    assert not info["errflag"]
    rhs2, _ = oracle.compute_lhs(d, f, out["u"], out["v"], out["w"], model=cfg["model"])
    assert np.sqrt(np.mean(rhs2 ** 2)) <= 1e-10 * np.sqrt(np.mean(out["rhs"] ** 2))
    # the step changed every field it owns (v stays when y_size = 1: pi'
    # is then uniform in y)
    for name_, before in (("u", u), ("v", v), ("w", w), ("rhop", rhop), ("pip", pip)):
        changed = rel_err(dom.interior(out[name_]), dom.interior(before)) > 1e-8
        assert changed == (name_ != "v" or dom.ny > 1), name_
