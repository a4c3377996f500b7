"""GPU parity: every kernel of the Poisson path against the CPU oracle.

Tolerances (relative to the largest magnitude of the oracle result):
  operator assembly FP64   1e-12  (same algebra, different association)
  operator apply FP64      1e-13
  operator apply FP32      2e-6   (FP32 operator copy, FP32 input)
  preconditioner FP64      1e-12
  preconditioner FP32      1e-4
  full solve (FP64)        iteration count within max(8, 15 %) of the oracle's
                           (BiCGSTAB counts at 1e-10 move by several iterations
                           under 1e-16 input perturbations); pressure within
                           1e-6 of the oracle's, both at relative residual 1e-10
"""
import numpy as np
import pytest

from _cases import CASES, case, consistent_rhs, iterations_agree, null_weights, oracle_operator, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solvers(pcf):
    cache = {}

    def get(name):
        if name not in cache:
            cfg = case(name)
            s = pcf.PoissonSolver(cfg["dom"], cfg["model"])
            s.set_grid(cfg["fields"])
            s.set_background(cfg["fields"])
            cache[name] = (cfg, s)
        return cache[name]

    yield get
    for _, s in cache.values():
        s.close()


def _drop_null(cfg, x):
    """Removes the component along the right null vector fcscal (a constant
    Exner-pressure offset), which the right-hand side does not determine."""
    dom = cfg["dom"]
    nv = null_weights(cfg) / dom.interior(cfg["fields"]["jac"])
    return x - np.vdot(nv, x) / np.vdot(nv, nv) * nv


@pytest.mark.parametrize("name", CASES)
def test_assembly_matches_oracle(name, solvers, oracle):
    cfg, s = solvers(name)
    _, ref = oracle_operator(oracle, cfg)
    got = s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["damp"], cfg["p"])
    assert np.isfinite(got).all()
    for c in range(25):
        scale = max(np.abs(ref).max(), 1e-300)
        err = np.abs(got[c] - ref[c]).max() / scale
        assert err < 1e-12, (name, oracle.COEF_NAMES[c], err)


@pytest.mark.parametrize("name", CASES)
def test_assembly_writes_every_operator_form(name, solvers):
    """The assembly writes the FP64, FP32 and difference-form FP32 operators
    (and fcscal) in one pass; uploading its FP64 planes with set_operator
    rebuilds the FP32 copy and the difference form from them.  Every form
    must come out the same either way: the applies agree bitwise."""
    cfg, s = solvers(name)
    coef = s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["damp"], cfg["p"])
    x = np.random.default_rng(8).standard_normal(cfg["dom"].interior_shape)
    forms = [("fp64", False), ("fp32", False), ("fp32", True), ("mixed", False)]
    fused = [s.apply_operator(x, horizontal=h, precision=p) for p, h in forms]
    s.set_operator(coef)
    rebuilt = [s.apply_operator(x, horizontal=h, precision=p) for p, h in forms]
    for (p, h), a, b in zip(forms, fused, rebuilt):
        assert np.array_equal(a, b), (name, p, h, np.abs(a - b).max())


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("horizontal", [False, True])
def test_apply_operator_matches_oracle(name, horizontal, solvers, oracle):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(cfg["dom"].interior_shape)
    ref = oracle.apply_operator(d, coef, x, horizontal)
    got = s.apply_operator(x, horizontal=horizontal, precision="fp64")
    assert rel_err(got, ref) < 1e-13
    got32 = s.apply_operator(x, horizontal=horizontal, precision="fp32")
    assert rel_err(got32, ref) < 2e-6


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("iters", [1, 2, 3])
def test_preconditioner_matches_oracle(name, iters, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    f = cfg["fields"]
    rng = np.random.default_rng(6)
    x = rng.standard_normal(cfg["dom"].interior_shape)
    nl = pcf.PoissonNamelist(preconditioner_iterations=iters, dtau=0.8)
    ref = oracle.apply_preconditioner(d, coef, f["dx"], f["dy"], 0.8, iters, x)
    got = s.apply_preconditioner(x, nl, precision="fp64")
    assert rel_err(got, ref) < 1e-12
    got32 = s.apply_preconditioner(x, nl, precision="fp32")
    assert rel_err(got32, ref) < 1e-4


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "rho", "comp"])
def test_global_dot(name, solvers, oracle):
    cfg, s = solvers(name)
    rng = np.random.default_rng(8)
    a = rng.standard_normal(cfg["dom"].interior_shape)
    b = rng.standard_normal(cfg["dom"].interior_shape)
    ref = oracle.dot(a, b)
    got = s.compute_global_dot_product(a, b)
    assert abs(got - ref) <= 1e-12 * np.abs(a * b).sum()
    # deterministic: bitwise identical on repeat
    assert s.compute_global_dot_product(a, b) == got


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "rho", "comp"])
def test_bicgstab_matches_oracle(name, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    f = cfg["fields"]
    rhs = consistent_rhs(oracle, cfg)
    ref, info_ref = oracle.bicgstab(d, coef, f["dx"], f["dy"], rhs, tolerance=1e-10, tolerance_is_relative=True,
                                    poisson_iterations=2000)
    nl = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=2000)
    got, info = s.apply_bicgstab(rhs, 1.0, nl)
    assert not info_ref["errflag"] and not info.errflag
    assert iterations_agree(info.niter, info_ref["niter"]), (info.niter, info_ref["niter"])
    assert info.residual <= 1e-10
    assert info.true_residual <= 2e-10
    assert rel_err(_drop_null(cfg, got), _drop_null(cfg, ref)) < 1e-6


@pytest.mark.parametrize("name", ["hill", "mtn", "rho", "comp"])
def test_solve_poisson_matches_oracle(name, solvers, oracle, pcf):
    cfg, s = solvers(name)
    dom = cfg["dom"]
    f = cfg["fields"]
    d = oracle.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=2000)
    rhs = consistent_rhs(oracle, cfg)
    ref, info_ref = oracle.solve_poisson(d, oracle.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], rhs,
                                         cfg["dt"], cfg["rayleigh_factor"], 1.0, cfg["damp"], cfg["p"], **kw)
    dpip = np.full(dom.halo_shape, -7.0)
    nl = pcf.PoissonNamelist(damp_horizontal_wind_on_rhs=cfg["damp"], **kw)
    info = s.solve_poisson(rhs, cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], 1.0, nl, dpip,
                           p=cfg["p"])
    assert not info.errflag and not info_ref["errflag"]
    assert iterations_agree(info.niter, info_ref["niter"]), (info.niter, info_ref["niter"])
    # halo cells untouched, interior written
    mask = np.ones(dom.halo_shape, bool)
    dom.interior(mask)[...] = False
    assert (dpip[mask] == -7.0).all()
    # dpip = s / fcscal / dt: its null-space component is a constant
    a, b = dom.interior(dpip), dom.interior(ref)
    assert rel_err(a - a.mean(), b - b.mean()) < 1e-6


@pytest.mark.parametrize("name", ["hill", "mtn", "rho"])
def test_mixed_precision_reaches_fp64_residual(name, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    rhs = consistent_rhs(oracle, cfg)
    nl = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000,
                             precision="mixed")
    got, info = s.apply_bicgstab(rhs, 1.0, nl)
    assert not info.errflag, info
    assert info.true_residual <= 1e-10
    # independent FP64 check of the residual with the oracle's operator
    r = rhs - oracle.apply_operator(d, coef, got)
    assert np.sqrt((r ** 2).mean()) / np.sqrt((rhs ** 2).mean()) <= 1.5e-10
    # the same solution as the plain FP64 solve, up to the solver tolerance
    ref, _ = oracle.bicgstab(d, coef, cfg["fields"]["dx"], cfg["fields"]["dy"], rhs, tolerance=1e-12,
                             tolerance_is_relative=True, poisson_iterations=4000)
    assert rel_err(_drop_null(cfg, got), _drop_null(cfg, ref)) < 1e-6


def test_error_paths(solvers, pcf):
    cfg, s = solvers("hill")
    dom = cfg["dom"]
    dpip = np.zeros(dom.halo_shape)
    nl = pcf.PoissonNamelist()
    with pytest.raises(ZeroDivisionError):
        s.solve_poisson(cfg["rhs"], cfg["rho"], cfg["betar"], 0.0, 1.0, 1.0, nl, dpip)
    # zero right-hand side: no iteration, dpip interior = 0 (apply_bicgstab!.jl:69-76)
    dpip[...] = 3.0
    info = s.solve_poisson(np.zeros(dom.interior_shape), cfg["rho"], cfg["betar"], cfg["dt"], 1.0, 1.0, nl, dpip)
    assert not info.errflag and info.niter == 0
    assert (dom.interior(dpip) == 0.0).all()
    # iteration cap: errflag, niter = poisson_iterations, dpip untouched
    dpip[...] = 3.0
    info = s.solve_poisson(cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], 1.0, 1.0,
                           pcf.PoissonNamelist(tolerance=1e-14, tolerance_is_relative=True, poisson_iterations=3),
                           dpip)
    assert info.errflag and info.niter == 3
    assert (dpip == 3.0).all()
    # non-finite input: reported, never a device fault
    bad = cfg["rhs"].copy()
    bad[0, 0, 0] = np.nan
    info = s.solve_poisson(bad, cfg["rho"], cfg["betar"], cfg["dt"], 1.0, 1.0, nl, dpip)
    assert info.errflag and info.status == pcf._lib.PCF_ENONFINITE
    # the context stays usable afterwards
    info = s.solve_poisson(cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], 1.0, 1.0, nl, dpip)
    assert not info.errflag


def test_bad_dims_rejected(pcf):
    from pincflow_poisson.fields import Domain
    with pytest.raises(pcf.PoissonError) as e:
        pcf.PoissonSolver(Domain(8, 8, 3))
    assert e.value.code == pcf._lib.PCF_EINVAL


def test_gpu_matches_golden_fixtures(pcf):
    """Against the committed oracle outputs (tests/golden/make_golden.py), no
    oracle run needed."""
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    from golden_cases import GOLDEN, golden_case
    gold = np.load(os.path.join(here, "golden", "small_cases.npz"))
    for name in GOLDEN:
        cfg = golden_case(name)
        with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
            s.set_grid(cfg["fields"])
            s.set_background(cfg["fields"])
            coef = s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["damp"],
                                      cfg["p"])
            assert rel_err(coef, gold[f"{name}/coef"]) < 1e-12, name
            x = np.random.default_rng(21).standard_normal(cfg["dom"].interior_shape)
            assert rel_err(s.apply_operator(x), gold[f"{name}/apply_total"]) < 1e-12
            assert rel_err(s.apply_operator(x, horizontal=True), gold[f"{name}/apply_horizontal"]) < 1e-12
            nl = pcf.PoissonNamelist(tolerance=1e-12, tolerance_is_relative=True)
            assert rel_err(s.apply_preconditioner(x, nl), gold[f"{name}/precond"]) < 1e-11
            sol, info = s.apply_bicgstab(gold[f"{name}/rhs"], 1.0, nl)
            assert not info.errflag
            assert rel_err(_drop_null(cfg, sol), _drop_null(cfg, gold[f"{name}/solution"])) < 1e-8


@pytest.mark.parametrize("name", ["hill", "mtn", "odd", "rho", "comp", "wide"])
def test_difference_form_fp32_operator(name, solvers, oracle):
    """The FP32 operator of the mixed solve (zero-row-sum difference form in
    pi = s / fcscal) applied to s equals A s to FP32 accuracy."""
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    x = np.random.default_rng(15).standard_normal(cfg["dom"].interior_shape)
    ref = oracle.apply_operator(d, coef, x)
    got = s.apply_operator(x, precision="mixed")
    assert rel_err(got, ref) < 5e-6
    if cfg["model"] == "Compressible":
        return  # dpdpi makes the compressible operator nonsingular
    # exact null space: A fcscal = 0 also in FP32
    from pincflow_poisson import fields as F
    fc = F.fcscal(cfg["dom"], cfg["fields"])
    a_fc = s.apply_operator(fc, precision="mixed")
    a_fc32 = s.apply_operator(fc, precision="fp32")
    scale = np.abs(coef[0]).max() * np.abs(fc).max()
    assert np.abs(a_fc).max() <= 1e-6 * scale
    assert np.abs(a_fc).max() <= np.abs(a_fc32).max()


def test_mixed_precision_iteration_count_at_scale(pcf):
    """On a stretched 128 x 96 x 48 mountain grid the reliable-update FP32 solve
    reaches the FP64 true residual 1e-10 within 25 % of the FP64 iteration count."""
    from pincflow_poisson import configs as C
    cfg = C.c2(nx=128, ny=96, nz=48)
    with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
        kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=5000, residual="true")
        _, i64 = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="fp64", **kw))
        x, imx = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="mixed", **kw))
        hist = s.residual_history()
    assert not i64.errflag and not imx.errflag, (i64, imx)
    assert imx.true_residual <= 1e-10
    assert imx.niter <= 1.25 * i64.niter + 5, (imx.niter, i64.niter)
    assert len(hist) == imx.niter and hist[-1] <= 1e-10


def test_tiny_grid_solves_in_one_block(solvers, oracle, pcf):
    """Grids of at most 2048 cells (the 40 x 1 x 40 periodic hill) run the
    reference FP64 BiCGSTAB in one thread block: a solve is a handful of
    launches (assembly, factors, the solve, the true residual), and its
    iteration count and solution match the oracle's as the multi-kernel path
    does; the mixed-precision setting gets the same FP64 solve."""
    cfg, s = solvers("hill")
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    rhs = consistent_rhs(oracle, cfg)
    ref, ri = oracle.bicgstab(d, coef, cfg["fields"]["dx"], cfg["fields"]["dy"], rhs, tolerance=1e-10,
                              tolerance_is_relative=True, poisson_iterations=4000)
    for prec in ("fp64", "mixed"):
        l0 = s.launch_count
        got, info = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True,
                                                                   poisson_iterations=4000, precision=prec,
                                                                   multigrid=prec == "mixed"))
        assert s.launch_count - l0 <= 6, s.launch_count - l0
        assert not info.errflag and iterations_agree(info.niter, ri["niter"]), (info.niter, ri["niter"])
        assert info.true_residual <= 1.01e-10
        assert rel_err(_drop_null(cfg, got), _drop_null(cfg, ref)) < 1e-6
        hist = s.residual_history()
        assert len(hist) == info.niter and hist[-1] <= 1e-10


@pytest.mark.parametrize("level", [0, 5, 31])
def test_staged_stencil_wait_gives_up_and_next_solve_succeeds(pcf, level):
    """The failure path of the TMA-staged V-cycle stencils: with the test hook
    the copy of one z-level is never issued (nothing is in flight for it) and
    every copy wait is bounded by 1 ms, so the wait runs out; the kernel drains
    its other copy, records PCF_ECUDA and leaves.  The solve reports errflag and
    status PCF_ECUDA without a device fault, dpip stays untouched, and with the
    hook off the next solve on the same handle converges to the same pressure
    as a fresh handle (the reduction state was reset)."""
    from pincflow_poisson import configs as C
    cfg = C.c2(nx=128, ny=64, nz=32)  # 128 wide: the finest level's stencils stage their tiles
    dom = cfg["dom"]
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=2000, residual="true",
              precision="mixed", multigrid=True)
    args = (cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["tolref"],
            pcf.PoissonNamelist(**kw))

    def handle():
        s = pcf.PoissonSolver(dom, cfg["model"])
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        return s

    with handle() as ref:
        good = np.zeros(dom.halo_shape)
        ok = ref.solve_poisson(*args, good)
        assert not ok.errflag
    with handle() as s:
        s.test_stall_staged_copy(level, 1e-3)
        dpip = np.full(dom.halo_shape, 3.0)
        info = s.solve_poisson(*args, dpip)
        assert info.errflag and info.status == pcf._lib.PCF_ECUDA, info
        assert (dpip == 3.0).all()
        s.test_stall_staged_copy(-1)
        again = s.solve_poisson(*args, dpip)
        assert not again.errflag and again.true_residual <= 1e-10, again
        assert again.niter == ok.niter
        inner, ref_inner = dom.interior(dpip), dom.interior(good)
        assert np.abs(inner - ref_inner).max() <= 1e-12 * np.abs(ref_inner).max()
