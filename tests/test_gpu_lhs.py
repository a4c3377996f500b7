"""GPU: compute_lhs! (pcf_compute_lhs, pcf_compute_lhs_device) against the
oracle's restatement (compute_lhs!.jl:68-223), and the device path from
winds to pressure.

Tolerances: rhs 1e-13 relative to its largest magnitude (the GPU multiplies
by reciprocals where the reference divides); tolref 1e-12."""
import numpy as np
import pytest

from _cases import case, rel_err
from pincflow_poisson import fields as F

pytestmark = pytest.mark.gpu


def _winds(dom, seed, walls=True):
    rng = np.random.default_rng(seed)
    u, v, w = (rng.standard_normal(dom.halo_shape) for _ in range(3))
    for a in (u, v, w):
        F._periodic_xy(dom, a)
    if walls:
        w[:dom.nbz] = 0.0
        w[dom.nbz + dom.nz - 1:] = 0.0
    return u, v, w


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "comp"])
def test_compute_lhs_matches_oracle(name, oracle, pcf):
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    u, v, w = _winds(dom, 21, walls=False)
    heat = np.random.default_rng(22).standard_normal(dom.interior_shape) if cfg["model"] == "Compressible" else None
    want, t_want = oracle.compute_lhs(d, f, u, v, w, model=cfg["model"], heating=heat)
    with pcf.PoissonSolver(dom, cfg["model"]) as s:
        s.set_grid(f)
        s.set_background(f)
        got, t_got = s.compute_lhs(u, v, w, heating=heat)
        z = np.zeros(dom.halo_shape)
        rhs0, t0 = s.compute_lhs(z, z, z)
    assert rel_err(got, want) < 1e-13, rel_err(got, want)
    assert abs(t_got - t_want) <= 1e-12 * abs(t_want)
    assert not rhs0.any() and t0 == 1.0


def test_device_path_from_winds_to_pressure(oracle, pcf):
    """compute_lhs_device writes the right-hand side straight into the solve's
    input; the pressure equals the host-array path's."""
    import torch
    cfg = case("mtn")
    dom, f = cfg["dom"], cfg["fields"]
    u, v, w = _winds(dom, 23)
    nl = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000,
                             precision="mixed", multigrid=True)
    with pcf.PoissonSolver(dom, cfg["model"]) as s:
        s.set_grid(f)
        s.set_background(f)
        rhs, tolref = s.compute_lhs(u, v, w)
        dp_host = np.zeros(dom.halo_shape)
        i1 = s.solve_poisson(rhs, cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], tolref, nl, dp_host)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        du, dv, dw, drho, dbr = t(u), t(v), t(w), t(cfg["rho"]), t(cfg["betar"])
        drhs = torch.zeros(dom.interior_shape, dtype=torch.float64, device="cuda")
        ddp = torch.zeros(dom.halo_shape, dtype=torch.float64, device="cuda")
        tol_dev = s.compute_lhs_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr(), drhs.data_ptr())
        i2 = s.solve_poisson_device(drhs.data_ptr(), drho.data_ptr(), dbr.data_ptr(), cfg["dt"],
                                    cfg["rayleigh_factor"], tol_dev, nl, ddp.data_ptr())
        dp_dev = ddp.cpu().numpy()
    assert tol_dev == tolref
    assert np.array_equal(drhs.cpu().numpy(), rhs)
    assert not i1.errflag and not i2.errflag and i1.niter == i2.niter
    assert np.array_equal(dp_dev, dp_host)
    # the divergence of winds with W = 0 at the walls is consistent: sum(J fcscal b) = 0
    wt = dom.interior(f["jac"]) * F.fcscal(dom, f)
    assert abs(np.sum(wt * rhs)) <= 1e-13 * np.sum(np.abs(wt * rhs))
