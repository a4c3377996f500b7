"""GPU: the pressure of the benchmark workloads against the oracle.

The oracle's plain FP64 BiCGSTAB (the reference algorithm,
apply_bicgstab!.jl:24-150, with the unscaling of solve_poisson!.jl:65-72)
was run to relative residual 1e-10 on the full 256 x 256 x 128 (c2) and
512 x 512 x 192 (c5) workloads, and on the first member of each size class of
the c4 ensemble, by tests/golden/make_oracle_iterations.py,
which committed a fingerprint of its converged pressure dpip: the values at
65,536 seeded interior cells, the mean, and the RMS of every z-level with the
mean removed.  Each test here solves the same workload through the host-array
entry point pcf_solve (PoissonSolver.solve_poisson) with the default method
(FP32 BiCGSTAB with the multigrid preconditioner inside FP64 refinement) and,
on c2, with the plain FP64 method; the c4 members are solved together by the
ensemble entry point on device arrays.

Both solves leave the constant (null-space) component of dpip free, so the
mean difference over the sampled cells is removed first.  Tolerances:
  max pointwise deviation at the sampled cells  <= 1e-6 of max |oracle - mean|
  per-level RMS (mean removed)                   <= 1e-6 relative, every level
  FP64 true relative residual                    <= 1e-10
"""
import os

import numpy as np
import pytest

from pincflow_poisson import configs as C

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KW = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000, residual="true")


def _fingerprint(name):
    p = os.path.join(HERE, "golden", f"{name}_fp64_fingerprint.npz")
    if not os.path.exists(p):
        pytest.skip(f"no oracle fingerprint for {name}")
    return np.load(p)


def _compare(fp, dpip):
    """(max pointwise deviation, max per-level RMS deviation), both relative."""
    ref = fp["values"]
    got = dpip.ravel()[fp["indices"]]
    diff = got - ref
    off = diff.mean()
    dev = float(np.abs(diff - off).max() / np.abs(ref - fp["mean"]).max())
    lv = np.sqrt(((dpip - dpip.mean()) ** 2).mean(axis=(1, 2)))
    lev = float(np.abs(lv - fp["level_rms"]).max() / fp["level_rms"].max())
    return dev, lev


def _solve(pcf, cfg, **nl):
    dom = cfg["dom"]
    with pcf.PoissonSolver(dom, cfg["model"]) as s:
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        dpip = np.zeros(dom.halo_shape)
        info = s.solve_poisson(cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"],
                               cfg["tolref"], pcf.PoissonNamelist(**KW, **nl), dpip)
    return dom.interior(dpip).copy(), info


@pytest.mark.parametrize("name,method", [("c2", "mg"), ("c2", "fp64"), ("c5", "mg")])
def test_pressure_matches_oracle_fingerprint(pcf, name, method):
    fp = _fingerprint(name)
    cfg = C.c2() if name == "c2" else C.c5()
    assert tuple(fp["shape"]) == cfg["dom"].interior_shape
    nl = dict(precision="fp64") if method == "fp64" else dict(precision="mixed", multigrid=True)
    dpip, info = _solve(pcf, cfg, **nl)
    assert not info.errflag
    assert info.true_residual <= 1e-10
    dev, lev = _compare(fp, dpip)
    print(f"{name} {method}: {info.niter} iterations (oracle {int(fp['niter'])}), true residual "
          f"{info.true_residual:.2e}, max pointwise deviation {dev:.2e}, level RMS {lev:.2e}")
    assert dev <= 1e-6
    assert lev <= 1e-6


def test_c4_ensemble_matches_oracle_fingerprints(pcf):
    """The 32-member c4 ensemble solved together (one graph launch for the
    whole iteration): the first member of each size class against the
    oracle's FP64 solve of that member (tests/golden/c4_<nx>_fp64_fingerprint.npz),
    same tolerances."""
    import torch
    sizes = C.c4_sizes()
    fps = {nx: _fingerprint(f"c4_{nx}") for nx in sorted(set(sizes))}
    nl = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000,
                             precision="mixed", multigrid=True, residual="true")
    members = []
    try:
        for q, nx in enumerate(sizes):
            cfg = C.c4(q, nx)
            s = pcf.PoissonSolver(cfg["dom"], cfg["model"])
            s.set_grid(cfg["fields"])
            s.set_background(cfg["fields"])
            dev = {k: torch.from_numpy(np.ascontiguousarray(cfg[k])).cuda() for k in ("rhs", "rho", "betar")}
            dev["dpip"] = torch.zeros(cfg["dom"].halo_shape, dtype=torch.float64, device="cuda")
            members.append((cfg, s, dev))
        with pcf.Ensemble([s for _, s, _ in members]) as ens:
            infos = ens.solve_poisson_device([d["rhs"].data_ptr() for _, _, d in members],
                                             [d["rho"].data_ptr() for _, _, d in members],
                                             [d["betar"].data_ptr() for _, _, d in members],
                                             [c["dt"] for c, _, _ in members],
                                             [c["rayleigh_factor"] for c, _, _ in members],
                                             [c["tolref"] for c, _, _ in members], nl,
                                             [d["dpip"].data_ptr() for _, _, d in members])
        for nx, fp in fps.items():
            q = sizes.index(nx)
            cfg, _, d = members[q]
            info = infos[q]
            assert not info.errflag and info.true_residual <= 1e-10, (nx, info)
            assert tuple(fp["shape"]) == cfg["dom"].interior_shape
            dpip = cfg["dom"].interior(d["dpip"].cpu().numpy())
            dev, lev = _compare(fp, dpip)
            print(f"c4 member {q} ({nx}^2): {info.niter} iterations (oracle {int(fp['niter'])}), "
                  f"max pointwise deviation {dev:.2e}, level RMS {lev:.2e}")
            assert dev <= 1e-6
            assert lev <= 1e-6
    finally:
        for _, s, _ in members:
            s.close()
