"""GPU: the multigrid preconditioner of the mixed solve against its oracle
(oracle/mg_oracle.py) and the plain FP64 solve.

Tolerances (relative to the largest magnitude of the oracle result):
  coarse operators      2e-5   (FP32 planes; levels >= 2 are built from FP32 inputs)
  one V-cycle           1e-4   (FP32 arithmetic through every level, with the
                               FP32 operator copy); the default BF16 copy of
                               the finest operator moves it by at most 2e-2,
                               and iteration counts stay within the rounding
                               noise of BiCGSTAB counts (max(8, 15 %), as
                               in _cases.iterations_agree)
  solve                 FP64 true residual <= 1e-10; pressure within 1e-6 of
                        the oracle's plain FP64 solution (null space removed)
"""
import numpy as np
import pytest

from _cases import CASES, case, consistent_rhs, iterations_agree, null_weights, oracle_operator, rel_err
from pincflow_poisson import fields as F

pytestmark = pytest.mark.gpu

MG = dict(multigrid=True, mg_dtau=2.0, mg_coarse_iterations=4, mg_min_columns=16)
# the parity cases plus one whose hierarchy aggregates 1 x 2 columns
MG_CASES = CASES + ["oddx", "wide2", "wide3"]


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
    dom = cfg["dom"]
    nv = null_weights(cfg) / dom.interior(cfg["fields"]["jac"])
    return x - np.vdot(nv, x) / np.vdot(nv, nv) * nv


def _oracle_mg(cfg, coef, **kw):
    from oracle.mg_oracle import Multigrid
    f = cfg["fields"]
    return Multigrid(coef, F.fcscal(cfg["dom"], f), f["dx"], f["dy"], dtau=kw.get("mg_dtau", 2.0),
                     coarse_iterations=kw.get("mg_coarse_iterations", 4), min_columns=kw.get("mg_min_columns", 16),
                     bf16_planes=kw.get("bf16_planes", False), fp8_smoother=kw.get("fp8_smoother", False))


def _fp8_active(cfg):
    """mg_smoother_fp8 takes effect where the finest level's copies are staged
    by TMA: rows of a multiple of 16 bytes in FP8, at least 128 wide."""
    nx = cfg["dom"].nx
    return nx % 16 == 0 and nx >= 128


@pytest.mark.parametrize("name", MG_CASES)
def test_hierarchy_and_coarse_operators(name, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    nl = pcf.PoissonNamelist(precision="mixed", **MG)
    levels = s.multigrid_levels(nl)
    mg = _oracle_mg(cfg, coef, **MG)
    assert levels == [l[:3] for l in mg.dims]
    for lv in range(1, min(4, len(levels))):
        got = s.multigrid_operator(lv, levels[lv])
        want = mg.levels[lv]["coef"]
        assert rel_err(got, want) < 2e-5, (lv, rel_err(got, want))


@pytest.mark.parametrize("name", MG_CASES)
def test_vcycle_matches_oracle(name, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    b = np.random.default_rng(17).standard_normal(cfg["dom"].interior_shape)
    got = s.apply_multigrid(b, pcf.PoissonNamelist(precision="mixed", mg_operator_bf16=False, **MG))
    want = _oracle_mg(cfg, coef, **MG).cycle(b)
    assert rel_err(got, want) < 1e-4, rel_err(got, want)
    # the BF16 operator copies (shared-memory staged stencils on wide grids)
    # against the oracle's V-cycle on the same BF16-rounded planes
    got16 = s.apply_multigrid(b, pcf.PoissonNamelist(precision="mixed", mg_smoother_fp8=False, **MG))
    want16 = _oracle_mg(cfg, coef, bf16_planes=True, **MG).cycle(b)
    assert rel_err(got16, want16) < 1e-4, rel_err(got16, want16)
    assert rel_err(got16, want) > 10 * rel_err(got16, want16), (rel_err(got16, want), rel_err(got16, want16))
    # mg_smoother_fp8: the finest level's pseudo-time steps on the FP8 copy
    # (where it is staged), against the oracle's V-cycle on the same FP8 planes
    got8 = s.apply_multigrid(b, pcf.PoissonNamelist(precision="mixed", mg_smoother_fp8=True, **MG))
    want8 = _oracle_mg(cfg, coef, bf16_planes=True, fp8_smoother=_fp8_active(cfg), **MG).cycle(b)
    assert rel_err(got8, want8) < 1e-4, rel_err(got8, want8)
    if _fp8_active(cfg):
        assert rel_err(got8, want16) > 10 * rel_err(got8, want8), (rel_err(got8, want16), rel_err(got8, want8))


@pytest.mark.parametrize("name", MG_CASES)
def test_fused_coarse_cycle_matches_oracle(name, solvers, oracle, pcf):
    """mg_fused_coarse: the levels of at most 1024 columns as one
    cooperative launch per cycle give the same V-cycle (FP32 and BF16 copies)
    and, on the parity cases, the same solve as one kernel per step."""
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    b = np.random.default_rng(17).standard_normal(cfg["dom"].interior_shape)
    for bf16 in (False, True):
        got = s.apply_multigrid(b, pcf.PoissonNamelist(precision="mixed", mg_operator_bf16=bf16,
                                                       mg_smoother_fp8=False, mg_fused_coarse=True, **MG))
        want = _oracle_mg(cfg, coef, bf16_planes=bf16, **MG).cycle(b)
        assert rel_err(got, want) < 1e-4, (bf16, rel_err(got, want))
    if name not in CASES:
        return  # wide3 takes 500-900 iterations either way: counts there are rounding noise
    rhs = consistent_rhs(oracle, cfg)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed", **MG)
    _, fused = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(mg_fused_coarse=True, **kw))
    _, steps = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(**kw))
    assert not fused.errflag and fused.true_residual <= 1e-10, fused
    assert iterations_agree(fused.niter, steps.niter), (fused.niter, steps.niter)


@pytest.mark.parametrize("dtau", [2.0, 2.5])
@pytest.mark.parametrize("name", CASES)
def test_multigrid_solve_reaches_fp64_residual(name, dtau, solvers, oracle, pcf):
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    s.set_operator(coef)
    rhs = consistent_rhs(oracle, cfg)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed")
    got, info = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(**kw, **dict(MG, mg_dtau=dtau)))
    assert not info.errflag, info
    assert info.true_residual <= 1e-10
    r = rhs - oracle.apply_operator(d, coef, got)
    assert np.sqrt((r ** 2).mean()) / np.sqrt((rhs ** 2).mean()) <= 1.5e-10
    ref, _ = oracle.bicgstab(d, coef, cfg["fields"]["dx"], cfg["fields"]["dy"], rhs, tolerance=1e-12,
                             tolerance_is_relative=True, poisson_iterations=4000)
    if cfg["model"] == "Compressible":
        assert rel_err(got, ref) < 1e-6
    else:
        assert rel_err(_drop_null(cfg, got), _drop_null(cfg, ref)) < 1e-6
    _, plain = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(**kw))
    assert info.niter <= plain.niter, (info.niter, plain.niter)


@pytest.mark.parametrize("name", CASES)
def test_bf16_operator_copy_keeps_the_iteration_count(name, solvers, oracle, pcf):
    """The finest level's V-cycle stencils read a BF16 copy of the operator
    by default; the copy follows every new operator (set_operator here, the
    assembly in solve_poisson)."""
    cfg, s = solvers(name)
    d, coef = oracle_operator(oracle, cfg)
    rhs = consistent_rhs(oracle, cfg)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed", **MG)
    for scale in (1.0, 0.5):  # a second operator on the same handle
        s.set_operator(coef * scale)
        _, i16 = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(**kw))
        _, i32 = s.apply_bicgstab(rhs, 1.0, pcf.PoissonNamelist(mg_operator_bf16=False, **kw))
        assert not i16.errflag and not i32.errflag and i16.true_residual <= 1e-10
        assert iterations_agree(i16.niter, i32.niter), (scale, i16.niter, i32.niter)


def test_fp8_smoother_keeps_the_iteration_count(pcf):
    """Stretched 128 x 96 x 48 mountain grid (the FP8 copy staged): the mixed
    solve with the finest level's pseudo-time steps on the FP8 copy reaches
    the FP64 true residual 1e-10 in the iterations of the BF16 copy (within
    the rounding noise of BiCGSTAB counts), and the same solution within 1e-6
    once the null-space component is removed."""
    from pincflow_poisson import configs as C
    cfg = C.c2(nx=128, ny=96, nz=48)
    with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
        kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, residual="true",
                  precision="mixed", **dict(MG, mg_dtau=2.5))
        x8, i8 = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(mg_smoother_fp8=True, **kw))
        x16, i16 = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(**kw))
    assert not i8.errflag and not i16.errflag and i8.true_residual <= 1e-10, (i8, i16)
    assert iterations_agree(i8.niter, i16.niter), (i8.niter, i16.niter)
    # the two solutions may differ by a multiple of the null vector fcscal
    assert rel_err(_drop_null(cfg, x8), _drop_null(cfg, x16)) < 1e-6


def test_multigrid_rejected_outside_the_mixed_solve(solvers, pcf):
    cfg, s = solvers("mtn")
    with pytest.raises(pcf.PoissonError) as e:
        s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="fp64", **MG))
    assert e.value.code == pcf._lib.PCF_EINVAL
    with pytest.raises(pcf.PoissonError) as e:
        s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="mixed", **dict(MG, mg_dtau=0.0)))
    assert e.value.code == pcf._lib.PCF_EINVAL


def test_multigrid_iteration_count_at_scale(pcf):
    """Stretched 128 x 96 x 48 mountain grid: the multigrid-preconditioned
    mixed solve reaches the FP64 true residual 1e-10 in at most a fifth of the
    plain FP64 iteration count."""
    from pincflow_poisson import configs as C
    cfg = C.c2(nx=128, ny=96, nz=48)
    with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
        kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=5000, residual="true")
        _, i64 = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="fp64", **kw))
        _, img = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(precision="mixed", **kw, **MG))
        hist = s.residual_history()
    assert not i64.errflag and not img.errflag, (i64, img)
    assert img.true_residual <= 1e-10
    assert 5 * img.niter <= i64.niter, (img.niter, i64.niter)
    assert len(hist) == img.niter and hist[-1] <= 1e-10
