"""GPU: batched solves of uneven ensemble members (pcf_ensemble_*) against
each member's own single-handle solve and the CPU oracle.

The ensemble runs the same device-side iteration as a single handle, so each
member's iteration count must equal its single-handle count and its pressure
agree to 1e-12 (relative to its largest magnitude); against the oracle's
plain FP64 solve the pressure agrees to 1e-6 (null space removed)."""
import numpy as np
import pytest

from _cases import rel_err

pytestmark = pytest.mark.gpu

SIZES = [32, 48, 64, 32, 40]
NL = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed",
          multigrid=True, residual="true")


@pytest.fixture(scope="module")
def members(pcf):
    import torch
    from pincflow_poisson import configs as C
    out = []
    for q, nx in enumerate(SIZES):
        cfg = C.c4(q, nx)
        if q == 3:
            cfg["rhs"] = np.zeros_like(cfg["rhs"])  # a member with nothing to solve
        s = pcf.PoissonSolver(cfg["dom"], cfg["model"])
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        dev = {k: torch.from_numpy(np.ascontiguousarray(cfg[k])).cuda() for k in ("rhs", "rho", "betar")}
        dev["dpip"] = torch.zeros(cfg["dom"].halo_shape, dtype=torch.float64, device="cuda")
        out.append((cfg, s, dev))
    yield out
    for _, s, _ in out:
        s.close()


def _solve_ensemble(pcf, ens, members, nl):
    return ens.solve_poisson_device([d["rhs"].data_ptr() for _, _, d in members],
                                    [d["rho"].data_ptr() for _, _, d in members],
                                    [d["betar"].data_ptr() for _, _, d in members],
                                    [c["dt"] for c, _, _ in members], [c["rayleigh_factor"] for c, _, _ in members],
                                    [c["tolref"] for c, _, _ in members], nl,
                                    [d["dpip"].data_ptr() for _, _, d in members])


@pytest.mark.parametrize("fused", [None, False])
def test_ensemble_matches_single_solves(pcf, members, fused):
    """fused None: the default, the coarse levels as one cluster launch in the
    ensemble; False: one kernel per step as in single solves."""
    nl = pcf.PoissonNamelist(**NL, mg_fused_coarse=fused)
    with pcf.Ensemble([s for _, s, _ in members]) as ens:
        infos = _solve_ensemble(pcf, ens, members, nl)
        got = [d["dpip"].cpu().numpy().copy() for _, _, d in members]
        # the same graph serves a second call
        infos2 = _solve_ensemble(pcf, ens, members, nl)
        again = [d["dpip"].cpu().numpy().copy() for _, _, d in members]
        assert ens.launch_count > 0
    for q, (cfg, s, d) in enumerate(members):
        info = infos[q]
        assert not info.errflag, (q, info)
        assert infos2[q].niter == info.niter
        assert rel_err(again[q], got[q]) <= 1e-12 if np.abs(got[q]).max() > 0 else np.abs(again[q]).max() == 0
        if q == 3:
            assert info.niter == 0 and np.abs(got[q]).max() == 0
            continue
        assert info.true_residual <= 1e-10
        d["dpip"].zero_()
        # the ensemble runs the coarse levels as one cluster launch by default
        # (mg_fused_coarse = -1); the single solve is asked for the same
        single = s.solve_poisson_device(d["rhs"].data_ptr(), d["rho"].data_ptr(), d["betar"].data_ptr(), cfg["dt"],
                                        cfg["rayleigh_factor"], cfg["tolref"],
                                        pcf.PoissonNamelist(**NL, mg_fused_coarse=fused is None),
                                        d["dpip"].data_ptr())
        ref = d["dpip"].cpu().numpy()
        assert single.niter == info.niter, (q, single.niter, info.niter)
        assert rel_err(got[q], ref) <= 1e-12, (q, rel_err(got[q], ref))


def test_ensemble_pressure_matches_oracle(pcf, oracle, members):
    from _cases import oracle_operator
    cfg, s, d = members[1]
    nl = pcf.PoissonNamelist(**NL)
    with pcf.Ensemble([m[1] for m in members]) as ens:
        infos = _solve_ensemble(pcf, ens, members, nl)
    assert not infos[1].errflag
    cfg = dict(cfg, damp=False, p=None)
    od, coef = oracle_operator(oracle, cfg)
    f = cfg["fields"]
    ref = oracle.solve_poisson(od, oracle.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["rhs"], cfg["dt"],
                               cfg["rayleigh_factor"], tolerance=1e-12, tolerance_is_relative=True,
                               poisson_iterations=4000)[0]
    dom = cfg["dom"]
    a, b = dom.interior(d["dpip"].cpu().numpy()), dom.interior(ref)
    assert rel_err(a - a.mean(), b - b.mean()) < 1e-6


def test_ensemble_with_autotuner(pcf, members):
    pcf.autotune_clear()
    nl = pcf.PoissonNamelist(**NL, autotune=True)
    with pcf.Ensemble([s for _, s, _ in members]) as ens:
        infos = _solve_ensemble(pcf, ens, members, nl)
    assert all(not i.errflag for i in infos)
    entries = pcf.autotune_entries()
    sizes = {(e["nx"], e["ny"], e["nz"]) for e in entries if e["kernel"] == "total32_diff"}
    assert sizes == {(nx, nx, nx // 2) for nx in set(SIZES)}
    for e in entries:
        assert e["tile_x"] in (32, 16, 8) and 2 <= e["levels"] <= e["nz"]
        if e["ms_default"] > 0:  # the heuristic shape is one of the candidates
            assert e["ms_best"] <= e["ms_default"]
    pcf.autotune_clear()


def test_ensemble_rejects_what_it_does_not_run(pcf, members):
    solvers = [s for _, s, _ in members]
    with pytest.raises(pcf.PoissonError):
        pcf.Ensemble([solvers[0], solvers[0]])
    with pcf.Ensemble(solvers) as ens:
        with pytest.raises(pcf.PoissonError) as e:
            _solve_ensemble(pcf, ens, members, pcf.PoissonNamelist(**dict(NL, precision="fp64", multigrid=False)))
        assert e.value.code == pcf._lib.PCF_EINVAL
