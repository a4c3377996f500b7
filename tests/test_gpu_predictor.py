"""GPU: the implicit half step around the solve against the oracle's
restatement (or_predict.cpp): set_boundaries!(BoundaryPredictands()),
modify_compressible_wind!, the implicit predictor (implicit_integration!.jl:
53-63) and the whole step (:49-77) with apply_corrector!.

Tolerances: the pointwise kernels 1e-12 relative to each field's largest
magnitude (FP64, the same operation order, but with FMA contraction; the GPU
squares dt by a product where the reference calls ^); the fill and the
compressible wind factors (explicitly rounded) bitwise.  The
whole step, whose solve stops at its own tolerance, as the corrector chain:
1e-6 relative to each field's change, dpip and pip without their constant."""
import numpy as np
import pytest

from _cases import CASES, case, rel_err
from pincflow_poisson import fields as F

pytestmark = pytest.mark.gpu


def _state(dom, seed, wkb=False):
    rng = np.random.default_rng(seed)
    u, v, w, rhop, pip = (rng.standard_normal(dom.halo_shape) for _ in range(5))
    rhop *= 1e-3
    tend = [1e-2 * rng.standard_normal(dom.halo_shape) for _ in range(2)] if wkb else [None, None]
    return u, v, w, rhop, pip, tend


def _dev(a):
    import torch
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return None if t is None else t.data_ptr()


def _solver(pcf, cfg):
    s = pcf.PoissonSolver(cfg["dom"], cfg["model"])
    s.set_grid(cfg["fields"])
    s.set_background(cfg["fields"])
    return s


@pytest.mark.parametrize("name", CASES)
def test_predictor_matches_oracle(name, oracle, pcf):
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    model = oracle.MODELS[cfg["model"]]
    u, v, w, rhop, pip, (dudt, dvdt) = _state(dom, 40, wkb=name in ("mtn", "comp"))
    want = oracle.implicit_predictor(d, model, f, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["rho"], rhop,
                                     u, v, w, pip, p=cfg["p"], dudt=dudt, dvdt=dvdt,
                                     damp_horizontal_wind_on_rhs=cfg["damp"])
    t = dict(u=_dev(u), v=_dev(v), w=_dev(w), rho=_dev(cfg["rho"]), rhop=_dev(rhop), pip=_dev(pip),
             p=_dev(cfg["p"]), betar=_dev(cfg["betar"]), dudt=_dev(dudt), dvdt=_dev(dvdt),
             wold=_dev(np.zeros(dom.halo_shape)))
    with _solver(pcf, cfg) as s:
        s.implicit_predictor_device(cfg["dt"], cfg["rayleigh_factor"], *[_ptr(t[k]) for k in
                                    ("u", "v", "w", "rho", "rhop", "pip", "betar")], d_p=_ptr(t["p"]),
                                    d_dudt=_ptr(t["dudt"]), d_dvdt=_ptr(t["dvdt"]), d_wold=_ptr(t["wold"]),
                                    damp_horizontal_wind_on_rhs=cfg["damp"])
    names = ("rho", "rhop", "u", "v", "w", "pip", "p", "wold")
    for label, x in zip(names, want):
        if x is None:
            continue
        g = t[label].cpu().numpy()
        assert rel_err(g, x) < 1e-12, (label, rel_err(g, x))


@pytest.mark.parametrize("model", ["Boussinesq", "PseudoIncompressible", "Compressible"])
def test_boundaries_and_wind_factors_match_oracle(model, oracle, pcf):
    cfg = case("comp")
    cfg["model"] = model
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    mi = oracle.MODELS[model]
    rng = np.random.default_rng(7)
    rho, rhop, u, v, w, pip = (rng.standard_normal(dom.halo_shape) for _ in range(6))
    p = cfg["p"]
    want = [a.copy() for a in (rho, rhop, u, v, w, pip, p)]
    oracle.modify_compressible_wind(d, mi, f, want[6], want[2], want[3], want[4])
    oracle.set_predictand_boundaries(d, mi, *want)
    back = [a.copy() for a in want]
    oracle.modify_compressible_wind(d, mi, f, back[6], back[2], back[3], back[4], divide=True)
    t = [_dev(a) for a in (rho, rhop, u, v, w, pip, p)]
    with _solver(pcf, cfg) as s:
        s.modify_compressible_wind_device(_ptr(t[6]), _ptr(t[2]), _ptr(t[3]), _ptr(t[4]))
        s.set_predictand_boundaries_device(*[_ptr(x) for x in t])
        got = [x.cpu().numpy() for x in t]
        s.modify_compressible_wind_device(_ptr(t[6]), _ptr(t[2]), _ptr(t[3]), _ptr(t[4]), divide=True)
        got_back = [x.cpu().numpy() for x in t]
    for label, g, x in zip(("rho", "rhop", "u", "v", "w", "pip", "p"), got, want):
        np.testing.assert_array_equal(g, x, err_msg=label)
    for label, g, x in zip(("u", "v", "w"), got_back[2:5], back[2:5]):
        np.testing.assert_array_equal(g, x, err_msg=label)


@pytest.mark.parametrize("name", ["mtn", "hill", "comp"])
def test_implicit_step_matches_oracle(name, oracle, pcf):
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    u, v, w, rhop, pip, _ = _state(dom, 41)
    for a in (u, v, w):
        F._periodic_xy(dom, a)
    want, winfo = oracle.implicit_step(d, cfg["model"], f, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"],
                                       cfg["rho"], rhop, u, v, w, pip, p=cfg["p"],
                                       damp_horizontal_wind_on_rhs=cfg["damp"], tolerance=1e-12,
                                       tolerance_is_relative=True, poisson_iterations=5000)
    assert not winfo["errflag"]
    nl = pcf.PoissonNamelist(tolerance=1e-11, tolerance_is_relative=True, poisson_iterations=5000,
                             damp_horizontal_wind_on_rhs=cfg["damp"])
    host = dict(u=u.copy(), v=v.copy(), w=w.copy(), rho=cfg["rho"].copy(), rhop=rhop.copy(), pip=pip.copy(),
                p=None if cfg["p"] is None else cfg["p"].copy(), dpip=np.zeros(dom.halo_shape),
                wold=np.zeros(dom.halo_shape))
    dev = {k: _dev(x) for k, x in host.items()}
    betar = _dev(cfg["betar"])
    with _solver(pcf, cfg) as s:
        info = s.implicit_step(cfg["dt"], cfg["rayleigh_factor"], nl, host["u"], host["v"], host["w"], host["rho"],
                               host["rhop"], host["pip"], cfg["betar"], host["dpip"], p=host["p"], wold=host["wold"])
        info_d = s.implicit_step_device(cfg["dt"], cfg["rayleigh_factor"], nl, *[_ptr(dev[k]) for k in
                                        ("u", "v", "w", "rho", "rhop", "pip")], _ptr(betar), _ptr(dev["dpip"]),
                                        d_p=_ptr(dev["p"]), d_wold=_ptr(dev["wold"]))
    assert not info.errflag and not info_d.errflag and info.niter == info_d.niter
    # host and device entry points run the same kernels on the same data
    for k, x in host.items():
        if x is not None:
            np.testing.assert_array_equal(dev[k].cpu().numpy(), x, err_msg=k)
    np.testing.assert_array_equal(host["wold"], want["wold"])
    for label in ("u", "v", "w", "rhop"):
        before = dict(u=u, v=v, w=w, rhop=rhop)[label]
        if dom.ny == 1 and label == "v":
            continue
        assert rel_err(host[label] - before, want[label] - before) < 1e-6, label
    for label, base in (("dpip", 0.0), ("pip", pip)):
        gi, xi = dom.interior(host[label] - base), dom.interior(want[label] - base)
        assert rel_err(gi - gi.mean(), xi - xi.mean()) < 1e-6, label
    np.testing.assert_array_equal(host["rho"], want["rho"])


def test_implicit_step_errflag_leaves_the_predicted_fields(oracle, pcf):
    cfg = case("mtn")
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    model = oracle.MODELS[cfg["model"]]
    u, v, w, rhop, pip, _ = _state(dom, 42)
    fields = [a.copy() for a in (cfg["rho"], rhop, u, v, w, pip)]
    oracle.set_predictand_boundaries(d, model, *fields, None)
    want = oracle.implicit_predictor(d, model, f, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], fields[0],
                                     fields[1], fields[2], fields[3], fields[4], fields[5])
    nl = pcf.PoissonNamelist(tolerance=1e-14, tolerance_is_relative=True, poisson_iterations=2)
    host = dict(u=u.copy(), v=v.copy(), w=w.copy(), rho=cfg["rho"].copy(), rhop=rhop.copy(), pip=pip.copy())
    with _solver(pcf, cfg) as s:
        info = s.implicit_step(cfg["dt"], cfg["rayleigh_factor"], nl, host["u"], host["v"], host["w"], host["rho"],
                               host["rhop"], host["pip"], cfg["betar"], np.zeros(dom.halo_shape))
        with pytest.raises(pcf.PoissonError):
            s.implicit_step(0.0, 1.0, nl, host["u"].copy(), host["v"].copy(), host["w"].copy(), host["rho"].copy(),
                            host["rhop"].copy(), host["pip"].copy(), cfg["betar"], np.zeros(dom.halo_shape))
    assert info.errflag
    for label, x in zip(("rho", "rhop", "u", "v", "w", "pip"), want[:6]):
        assert rel_err(host[label], x) < 1e-12, label
