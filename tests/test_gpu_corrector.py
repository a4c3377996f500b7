"""GPU: the corrector after the solve (pcf_correct, pcf_correct_device) and
the whole apply_corrector! chain (pcf_apply_corrector_device) against the
oracle's restatement of apply_corrector!.jl:44-61 / correct!.jl:164-385.

Tolerances: the corrector alone 1e-12 relative to each field's largest
magnitude (the GPU multiplies by reciprocals where the reference divides);
the chain, whose solve stops at 1e-10 (mixed precision with multigrid) while
the oracle's runs to 1e-12, 1e-6 relative to each field's change (dpip and
pip without their free constant), and the corrected winds' compute_lhs!
below 1e-9 of the uncorrected one."""
import numpy as np
import pytest

from _cases import CASES, case, rel_err
from pincflow_poisson import fields as F

pytestmark = pytest.mark.gpu


def _fields(dom, seed):
    rng = np.random.default_rng(seed)
    out = [rng.standard_normal(dom.halo_shape) for _ in range(6)]  # dpip, u, v, w, rhop, pip
    for a in out[1:4]:
        F._periodic_xy(dom, a)
    return out


@pytest.mark.parametrize("name", CASES)
def test_correct_matches_oracle(name, oracle, pcf):
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    dpip, u, v, w, rhop, pip = _fields(dom, 31)
    want = oracle.correct(d, oracle.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                          cfg["rayleigh_factor"], dpip, u, v, w, rhop, pip,
                          damp_horizontal_wind_on_rhs=cfg["damp"], p=cfg["p"])
    with pcf.PoissonSolver(dom, cfg["model"]) as s:
        s.set_grid(f)
        s.set_background(f)
        # the corrector reads rho, betar and p of the last solve
        z = np.zeros(dom.interior_shape)
        dz = np.zeros(dom.halo_shape)
        s.solve_poisson(z, cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], 1.0,
                        pcf.PoissonNamelist(), dz, p=cfg["p"])
        got = [a.copy() for a in (dpip, u, v, w, rhop, pip)]
        s.correct(cfg["dt"], cfg["rayleigh_factor"], *got, damp_horizontal_wind_on_rhs=cfg["damp"])
    for label, g, x in zip(("dpip", "u", "v", "w", "rhop", "pip"), got, want):
        assert rel_err(g, x) < 1e-12, (label, rel_err(g, x))


def test_apply_corrector_chain(oracle, pcf):
    import torch
    cfg = case("mtn")
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    _, u, v, w, rhop, pip = _fields(dom, 32)
    w[:dom.nbz] = 0.0
    w[dom.nbz + dom.nz - 1:] = 0.0
    model = oracle.MODELS[cfg["model"]]
    rhs, tolref = oracle.compute_lhs(d, f, u, v, w, model=cfg["model"])
    dp_ref, _ = oracle.solve_poisson(d, model, f, cfg["rho"], cfg["betar"], rhs, cfg["dt"], cfg["rayleigh_factor"],
                                     tolref=tolref, tolerance=1e-12, tolerance_is_relative=True,
                                     poisson_iterations=5000)
    want = oracle.correct(d, model, f, cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], dp_ref, u, v, w,
                          rhop, pip)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    dev = [t(a) for a in (u, v, w, cfg["rho"], rhop, cfg["betar"], pip)]
    ddp = torch.zeros(dom.halo_shape, dtype=torch.float64, device="cuda")
    nl = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed",
                             multigrid=True)
    with pcf.PoissonSolver(dom, cfg["model"]) as s:
        s.set_grid(f)
        s.set_background(f)
        info = s.apply_corrector_device(*[x.data_ptr() for x in dev], cfg["dt"], cfg["rayleigh_factor"], nl,
                                        ddp.data_ptr())
        got = [x.cpu().numpy() for x in (ddp, dev[0], dev[1], dev[2], dev[4], dev[6])]
        rhs2, _ = s.compute_lhs(got[1], got[2], got[3])
    assert not info.errflag and info.true_residual <= 1e-10
    # corrections of the winds and rho' depend on dpip's gradients only; dpip
    # and pip's change are compared without their constant (null-space) part
    for label, g, x, b in zip(("u", "v", "w", "rhop"), got[1:5], want[1:5], (u, v, w, rhop)):
        assert rel_err(g - b, x - b) < 1e-6, (label, rel_err(g - b, x - b))
    for label, g, x, b in (("dpip", got[0], want[0], 0.0), ("pip", got[5], want[5], pip)):
        gi, xi = dom.interior(g - b), dom.interior(x - b)
        assert rel_err(gi - gi.mean(), xi - xi.mean()) < 1e-6, label
    assert np.sqrt(np.mean(rhs2 ** 2)) <= 1e-9 * np.sqrt(np.mean(rhs ** 2))
