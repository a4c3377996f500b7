"""CPU: the oracle against known answers, and the product's input generators
against the oracle.  No GPU.

The reference ships no golden vectors for its Poisson path (its only pinned
numbers are end-to-end norms of whole simulations) and Julia is absent, so
the oracle is pinned by analytic known-answer tests:
  * flat terrain: the operator is the separable 7-point Laplacian
    d_xx + d_yy + d_zz / (1 + N^2 dt^2) with Neumann walls, whose Fourier-cosine
    eigenpairs are known in closed form;
  * the null vectors implied by the divergence form (A fcscal = 0 and
    sum(J fcscal A s) = 0 when rho' = 0);
  * manufactured solutions, dense tridiagonal solves, linearity;
and by committed fixtures (tests/golden/) that pin it against drift.
"""
import json
import os

import numpy as np
import pytest

from _cases import case, oracle_operator, rel_err
from pincflow_poisson import configs as C
from pincflow_poisson import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))


def _flat(nx, ny, nz, nbv=0.012, dt=0.8):
    dom = F.Domain(nx, ny, nz)
    lx, ly, lz = 30e3, 20e3, 10e3
    g = F.grid(dom, lx, ly, lz, np.zeros((ny, nx)))
    atm = F.atmosphere_stable(dom, nbv, 300.0)
    f = dict(g)
    f.update(atm)
    return dom, f, dt


def test_constants_match_reference_values(oracle):
    c = oracle.constants()
    p = F.constants()
    for k in c:
        assert c[k] == pytest.approx(p[k], rel=1e-15)
    # Constants.jl:119-155: Ma = Fr = 1, kappa = 2/7
    assert c["ma"] == 1.0 and c["sig"] == pytest.approx(1.0)
    assert c["kappa"] == pytest.approx(0.4 / 1.4)


@pytest.mark.parametrize("which", ["c1", "c2_small", "c3_small", "c5_small"])
def test_generators_match_oracle(which, oracle):
    if which == "c1":
        cfg, L, st = C.c1(), (20000.0, 1000.0, 20000.0), 1.0
    elif which == "c2_small":
        cfg, L, st = C.c2(nx=20, ny=12, nz=10), (100e3, 100e3, 20e3), 1.5
    elif which == "c3_small":
        cfg, L, st = C.c3(5, nx=16, ny=16, nz=8), (100e3, 100e3, 20e3), 1.0
    else:
        cfg, L, st = C.c5(nx=16, ny=16, nz=12), (400e3, 400e3, 40e3), 1.0
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    hb = f["hb"][dom.nby:dom.nby + dom.ny, dom.nbx:dom.nbx + dom.nx] * F.constants()["lref"]
    g = oracle.grid(d, *L, st, np.ascontiguousarray(hb))
    for k in ("jac", "met13", "met23", "met33", "zc"):
        assert rel_err(f[k], g[k]) < 1e-14, k
    if cfg["model"] == "Boussinesq":
        nbv = np.sqrt(f["n2"].flat[0]) / F.constants()["tref"]
        a = oracle.atmosphere(d, 0, [nbv, 300.0], g["jac"], g["zc"], g["dz"])
    else:
        a = oracle.atmosphere(d, 1, [250.0, 1e5], g["jac"], g["zc"], g["dz"])
    for k in ("pbar", "rhobar", "thetabar", "n2"):
        assert rel_err(f[k], a[k]) < 1e-13, k
    if which == "c1":
        b = oracle.sponge_sin2(d, g["zc"], 10000.0, 20000.0, cfg["dt"])
        assert rel_err(cfg["betar"], b) < 1e-14


@pytest.mark.parametrize("m,n,l", [(1, 0, 1), (2, 1, 3), (0, 2, 5), (3, 3, 2), (1, 1, 0)])
def test_flat_terrain_fourier_eigenpairs(m, n, l, oracle):
    nx, ny, nz = 12, 10, 8
    dom, f, dt = _flat(nx, ny, nz)
    d = oracle.dims(nx, ny, nz)
    z = np.zeros(dom.halo_shape)
    coef = oracle.compute_operator(d, 0, f, z, z, dt, 1.0)
    i, j, k = np.arange(nx), np.arange(ny), np.arange(nz)
    s = (np.cos(np.pi * l * (k + 0.5) / nz)[:, None, None] * np.cos(2 * np.pi * n * j / ny)[None, :, None]
         * np.cos(2 * np.pi * m * i / nx)[None, None, :])
    cfac = 1.0 / (1.0 + f["n2"].flat[0] * dt ** 2)
    lam = (-(2 - 2 * np.cos(2 * np.pi * m / nx)) / f["dx"] ** 2 - (2 - 2 * np.cos(2 * np.pi * n / ny)) / f["dy"] ** 2
           - cfac * (2 - 2 * np.cos(np.pi * l / nz)) / f["dz"] ** 2)
    As = oracle.apply_operator(d, coef, s)
    scale = np.abs(coef[0]).max() * np.abs(s).max()
    assert np.abs(As - lam * s).max() <= 1e-12 * scale
    # cross terms vanish on flat terrain
    for name in ("ald", "alu", "ard", "aru", "abd", "abu", "afd", "afu", "add", "auu", "aldd", "aluu", "ardd",
                 "aruu", "abdd", "abuu", "afdd", "afuu"):
        assert np.abs(coef[oracle.COEF_NAMES.index(name)]).max() <= 1e-14 * np.abs(coef[0]).max(), name


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "wide"])
def test_null_vectors(name, oracle):
    cfg = case(name)
    d, coef = oracle_operator(oracle, cfg)
    dom, f = cfg["dom"], cfg["fields"]
    fc = F.fcscal(dom, f)
    Afc = oracle.apply_operator(d, coef, fc)
    assert np.abs(Afc).max() <= 1e-13 * np.abs(coef[0]).max() * np.abs(fc).max()
    w = dom.interior(f["jac"]) * fc
    s = np.random.default_rng(3).standard_normal(dom.interior_shape)
    As = oracle.apply_operator(d, coef, s)
    assert abs(np.sum(w * As)) <= 1e-14 * np.sum(np.abs(w * As))


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "rho", "comp"])
def test_manufactured_solution(name, oracle):
    cfg = case(name)
    d, coef = oracle_operator(oracle, cfg)
    dom, f = cfg["dom"], cfg["fields"]
    xs = np.random.default_rng(4).standard_normal(dom.interior_shape)
    b = oracle.apply_operator(d, coef, xs)
    sol, info = oracle.bicgstab(d, coef, f["dx"], f["dy"], b, tolerance=1e-12, tolerance_is_relative=True,
                                poisson_iterations=3000)
    assert not info["errflag"]
    nv = F.fcscal(dom, f)

    def drop(x):
        return x - np.vdot(nv, x) / np.vdot(nv, nv) * nv

    assert rel_err(drop(sol), drop(xs)) < 1e-7


@pytest.mark.parametrize("name", ["mtn", "comp"])
def test_thomas_sweep_equals_dense_tridiagonal_solve(name, oracle):
    cfg = case(name)
    d, coef = oracle_operator(oracle, cfg)
    dom, f = cfg["dom"], cfg["fields"]
    dtau = 0.9
    deta = dtau / (2 * (1 / f["dx"] ** 2 + 1 / f["dy"] ** 2))
    b = np.random.default_rng(5).standard_normal(dom.interior_shape)
    got = oracle.apply_preconditioner(d, coef, f["dx"], f["dy"], dtau, 1, b)
    ac, ad, au = coef[0], coef[5], coef[6]
    ref = np.empty_like(b)
    for j in range(dom.ny):
        for i in range(dom.nx):
            T = np.diag(1 - deta * ac[:, j, i]) - np.diag(deta * ad[1:, j, i], -1) - np.diag(deta * au[:-1, j, i], 1)
            ref[:, j, i] = np.linalg.solve(T, -deta * b[:, j, i])
    assert rel_err(got, ref) < 1e-12


def test_preconditioner_is_linear(oracle):
    cfg = case("mtn")
    d, coef = oracle_operator(oracle, cfg)
    f = cfg["fields"]
    rng = np.random.default_rng(6)
    a = rng.standard_normal(cfg["dom"].interior_shape)
    b = rng.standard_normal(cfg["dom"].interior_shape)
    M = lambda x: oracle.apply_preconditioner(d, coef, f["dx"], f["dy"], 1.0, 2, x)  # noqa: E731
    assert rel_err(M(2.5 * a + b), 2.5 * M(a) + M(b)) < 1e-12


def test_compute_lhs_is_consistent(oracle):
    """compute_lhs! of any staggered velocity is a divergence: sum(J fcscal b) = 0
    when the wall-normal velocity vanishes at the walls; zero velocity gives
    b = 0 and tolref = 1 (compute_lhs!.jl:149-157)."""
    cfg = C.c2(nx=16, ny=12, nz=8)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    rng = np.random.default_rng(7)
    u, v, w = (rng.standard_normal(dom.halo_shape) for _ in range(3))
    for a in (u, v, w):
        F._periodic_xy(dom, a)
    w[:dom.nbz] = 0.0
    w[dom.nbz + dom.nz - 1:] = 0.0
    rhs, tolref = oracle.compute_lhs(d, f, u, v, w)
    wt = dom.interior(f["jac"]) * F.fcscal(dom, f)
    assert abs(np.sum(wt * rhs)) <= 1e-13 * np.sum(np.abs(wt * rhs))
    assert 0 < tolref < 10
    z = np.zeros(dom.halo_shape)
    rhs0, t0 = oracle.compute_lhs(d, f, z, z, z)
    assert not rhs0.any() and t0 == 1.0


def test_solve_poisson_error_paths(oracle):
    cfg = C.c1()
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    with pytest.raises(ZeroDivisionError):
        oracle.solve_poisson(d, 0, f, cfg["rho"], cfg["betar"], cfg["rhs"], 0.0, 1.0)
    dp, info = oracle.solve_poisson(d, 0, f, cfg["rho"], cfg["betar"], np.zeros(dom.interior_shape), cfg["dt"], 1.0)
    assert info["niter"] == 0 and not info["errflag"] and not dp.any()
    _, info = oracle.solve_poisson(d, 0, f, cfg["rho"], cfg["betar"], cfg["rhs"], cfg["dt"], 1.0, tolerance=1e-14,
                                   tolerance_is_relative=True, poisson_iterations=4)
    assert info["errflag"] and info["niter"] == 4


def test_oracle_matches_golden_fixtures(oracle):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from golden_cases import GOLDEN, golden_case
    gold = np.load(os.path.join(HERE, "golden", "small_cases.npz"))
    for name in GOLDEN:
        cfg = golden_case(name)
        dom, f = cfg["dom"], cfg["fields"]
        d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
        coef = oracle.compute_operator(d, oracle.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                                       cfg["rayleigh_factor"], cfg["damp"], cfg["p"])
        assert rel_err(coef, gold[f"{name}/coef"]) < 1e-13
        x = np.random.default_rng(21).standard_normal(dom.interior_shape)
        assert rel_err(oracle.apply_operator(d, coef, x), gold[f"{name}/apply_total"]) < 1e-13
        assert rel_err(oracle.apply_operator(d, coef, x, True), gold[f"{name}/apply_horizontal"]) < 1e-13
        assert rel_err(oracle.apply_preconditioner(d, coef, f["dx"], f["dy"], 1.0, 2, x),
                       gold[f"{name}/precond"]) < 1e-12


@pytest.mark.parametrize("config, lo, hi", [("c2", 300, 700), ("c5", 600, 1200)])
def test_oracle_iteration_fixtures_are_converged(config, lo, hi):
    """The oracle's full FP64 solves behind bench.py's CPU baselines
    (tests/golden/make_oracle_iterations.py) reached 1e-10."""
    with open(os.path.join(HERE, "golden", f"{config}_fp64_oracle.json")) as fh:
        d = json.load(fh)
    assert not d["errflag"] and d["true_residual"] <= 1e-10 and lo < d["niter"] < hi


FINGERPRINTS = ["c2", "c5", "c4_64", "c4_96", "c4_128", "c4_192"]


@pytest.mark.parametrize("name", FINGERPRINTS)
def test_fingerprints_agree_with_their_records(name):
    """Every committed fingerprint of an oracle solve (the parity target of
    tests/test_gpu_baseline.py) belongs to the recorded full solve: same
    iteration count and true residual, distinct in-range sample indices."""
    fp = np.load(os.path.join(HERE, "golden", f"{name}_fp64_fingerprint.npz"))
    config = name.split("_")[0]
    with open(os.path.join(HERE, "golden", f"{config}_fp64_oracle.json")) as fh:
        rec = json.load(fh)
    if config == "c4":
        rec = rec["classes"][name.split("_")[1]]
    assert int(fp["niter"]) == rec["niter"] and float(fp["true_residual"]) == rec["true_residual"] <= 1e-10
    n = int(np.prod(fp["shape"]))
    idx = fp["indices"]
    assert len(np.unique(idx)) == len(idx) == min(65536, n) and idx.min() >= 0 and idx.max() < n
    assert fp["level_rms"].shape == (int(fp["shape"][0]),) and np.all(fp["level_rms"] > 0)


def test_oracle_reproduces_the_smallest_c4_fingerprint(oracle):
    """The oracle's FP64 solve of the 64 x 64 x 32 c4 member (about 1 s)
    reproduces its committed fingerprint bitwise: the oracle behind the
    full-size parity targets has not drifted."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_oracle_iterations import fingerprint_indices
    fp = np.load(os.path.join(HERE, "golden", "c4_64_fp64_fingerprint.npz"))
    sizes = C.c4_sizes()
    q = sizes.index(64)
    cfg = C.c4(q, 64)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    coef = oracle.compute_operator(d, oracle.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                                   cfg["rayleigh_factor"])
    sol, info = oracle.bicgstab(d, coef, f["dx"], f["dy"], cfg["rhs"], tolerance=1e-10, tolerance_is_relative=True,
                                poisson_iterations=5000)
    assert info["niter"] == int(fp["niter"])
    pb, rb = dom.interior(f["pbar"]), dom.interior(f["rhobar"])
    dpip = sol / np.sqrt(pb * pb / rb) / cfg["dt"]
    idx = fingerprint_indices(dpip.size)
    assert np.array_equal(idx, fp["indices"])
    assert np.array_equal(dpip.ravel()[idx], fp["values"])


def test_network_oracle_gradient_matches_finite_differences():
    """Pins the network oracle: its analytic gradient (exact float64 network)
    against central differences along random directions."""
    from oracle import net_oracle as NO
    rng = np.random.default_rng(0)
    d = {}
    for name, shape in NO.SIZES:
        d[name] = rng.standard_normal(shape) * (0.2 if name.startswith("W") else 0.05)
    p = NO.pack(d)
    b = rng.standard_normal((64, 4, 5))
    x = rng.standard_normal((64, 4, 5))
    _, g = NO.loss_and_grad(p, b, x, bf=False)
    for k in range(3):
        v = rng.standard_normal(p.size)
        eps = 1e-6
        lp, _ = NO.loss_and_grad(p + eps * v, b, x, bf=False)
        lm, _ = NO.loss_and_grad(p - eps * v, b, x, bf=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-5 * max(1.0, abs(fd)), (fd, g @ v)


def test_compute_lhs_compressible_is_a_flux_divergence(oracle):
    """Compressible compute_lhs! (compute_lhs!.jl:162-223): with periodic mass
    fluxes and W = 0 at the walls, sum(J fcscal b) = -kappa sum(J heating)
    (Ma = 1), i.e. 0 without heating; zero fluxes and heating give b = 0,
    tolref = 1."""
    cfg = C.c2(nx=16, ny=12, nz=8)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    rng = np.random.default_rng(8)
    u, v, w = (rng.standard_normal(dom.halo_shape) for _ in range(3))
    for a in (u, v, w):
        F._periodic_xy(dom, a)
    w[:dom.nbz] = 0.0
    w[dom.nbz + dom.nz - 1:] = 0.0
    wt = dom.interior(f["jac"]) * F.fcscal(dom, f)
    kappa = oracle.constants()["kappa"]
    rhs, tolref = oracle.compute_lhs(d, f, u, v, w, model="Compressible")
    assert abs(np.sum(wt * rhs)) <= 1e-13 * np.sum(np.abs(wt * rhs)) and 0 < tolref < 10
    heat = np.full(dom.interior_shape, 0.3)
    rhs_h, _ = oracle.compute_lhs(d, f, u, v, w, model="Compressible", heating=heat)
    want = -kappa * 0.3 * np.sum(dom.interior(f["jac"]))
    assert abs(np.sum(wt * rhs_h) - want) <= 1e-12 * abs(want)
    z = np.zeros(dom.halo_shape)
    rhs0, t0 = oracle.compute_lhs(d, f, z, z, z, model="Compressible")
    assert not rhs0.any() and t0 == 1.0


@pytest.mark.parametrize("name", ["mtn", "hill", "odd"])
def test_corrector_removes_the_divergence(name, oracle):
    """The reference's projection: compute_lhs! -> solve_poisson! -> correct!
    leaves winds whose compute_lhs! vanishes (to the solver tolerance), which
    ties the restatements of the operator, compute_lhs! and correct! (with
    compute_pressure_gradient and the dpip halo fill) to one another."""
    from _cases import case
    cfg = case(name)
    dom, f = cfg["dom"], cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    rng = np.random.default_rng(3)
    u, v, w = (rng.standard_normal(dom.halo_shape) for _ in range(3))
    for a in (u, v, w):
        F._periodic_xy(dom, a)
    w[:dom.nbz] = 0.0
    w[dom.nbz + dom.nz - 1:] = 0.0
    model = oracle.MODELS[cfg["model"]]
    rhs, tolref = oracle.compute_lhs(d, f, u, v, w, model=cfg["model"])
    dpip, info = oracle.solve_poisson(d, model, f, cfg["rho"], cfg["betar"], rhs, cfg["dt"], cfg["rayleigh_factor"],
                                      tolref=tolref, tolerance=1e-13, tolerance_is_relative=True,
                                      poisson_iterations=5000)
    assert not info["errflag"]
    z = np.zeros(dom.halo_shape)
    _, u2, v2, w2, _, _ = oracle.correct(d, model, f, cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"],
                                         dpip, u, v, w, z, z)
    rhs2, _ = oracle.compute_lhs(d, f, u2, v2, w2, model=cfg["model"])
    assert np.sqrt(np.mean(rhs2 ** 2)) <= 1e-11 * np.sqrt(np.mean(rhs ** 2))
