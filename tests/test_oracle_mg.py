"""CPU: the multigrid oracle (oracle/mg_oracle.py) against the properties its
algorithm guarantees, on small seeded cases."""
import numpy as np
import pytest

from _cases import case, oracle_operator
from pincflow_poisson import fields as F


@pytest.fixture(scope="module")
def mtn(oracle):
    cfg = case("mtn")
    d, coef = oracle_operator(oracle, cfg)
    return cfg, coef


def test_level_dims_rule():
    from oracle.mg_oracle import level_dims
    assert [l[:2] for l in level_dims(256, 256, 8, 16)] == [(256, 256), (128, 128), (64, 64), (32, 32), (16, 16),
                                                             (8, 8), (4, 4)]
    assert [l[:2] for l in level_dims(40, 1, 8, 16)] == [(40, 1), (20, 1), (10, 1)]
    assert [l[:2] for l in level_dims(96, 96, 8, 16)] == [(96, 96), (48, 48), (24, 24), (12, 12), (6, 6), (3, 3)]
    assert [l[:2] for l in level_dims(37, 29, 8, 16)] == [(37, 29)]
    assert [l[3:] for l in level_dims(48, 40, 8, 16)] == [(1, 1), (2, 2), (2, 2), (2, 2), (2, 1)]


def test_coarse_operator_keeps_the_null_space(mtn):
    """A fcscal = 0 on the finest level (rho' = 0) carries over: every coarse
    operator annihilates its own fcscal (row sums of the unscaled operator are
    aggregated and the face re-scaling moves weight within a row)."""
    from oracle.mg_oracle import apply, coarsen
    cfg, coef = mtn
    fc = F.fcscal(cfg["dom"], cfg["fields"])
    assert np.abs(apply(coef, fc)).max() <= 1e-10 * np.abs(coef).max()
    c, f = coef, fc
    for cx, cy in [(2, 2), (2, 2), (2, 1)]:
        c, f = coarsen(c, f, cx, cy)
        assert np.abs(apply(c, f)).max() <= 1e-10 * np.abs(c).max()


def test_coarse_operator_of_a_flat_laplacian_is_the_rediscretisation():
    """Constant-coefficient 5-point x-y Laplacian (no z coupling): the coarse
    operator equals the same stencil on the doubled grid spacing."""
    from oracle.mg_oracle import INDEX, coarsen
    nz, ny, nx = 4, 8, 8
    coef = np.zeros((25, nz, ny, nx))
    hx, hy = 2.0, 3.0
    coef[INDEX[(-1, 0, 0)]] = coef[INDEX[(1, 0, 0)]] = 1 / hx ** 2
    coef[INDEX[(0, -1, 0)]] = coef[INDEX[(0, 1, 0)]] = 1 / hy ** 2
    coef[0] = -2 / hx ** 2 - 2 / hy ** 2
    c, _ = coarsen(coef, np.ones((nz, ny, nx)), 2, 2)
    assert np.allclose(c[INDEX[(1, 0, 0)]], 1 / (2 * hx) ** 2)
    assert np.allclose(c[INDEX[(0, -1, 0)]], 1 / (2 * hy) ** 2)
    assert np.allclose(c[0], -2 / (2 * hx) ** 2 - 2 / (2 * hy) ** 2)
    others = [p for p in range(25) if p not in (0, INDEX[(1, 0, 0)], INDEX[(-1, 0, 0)], INDEX[(0, 1, 0)],
                                                 INDEX[(0, -1, 0)])]
    assert np.abs(c[others]).max() == 0


def test_vcycle_is_linear(mtn):
    from oracle.mg_oracle import Multigrid
    cfg, coef = mtn
    f = cfg["fields"]
    mg = Multigrid(coef, F.fcscal(cfg["dom"], f), f["dx"], f["dy"], dtau=2.0)
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal((2,) + cfg["dom"].interior_shape)
    lhs = mg.cycle(2.5 * a + b)
    rhs = 2.5 * mg.cycle(a) + mg.cycle(b)
    assert np.abs(lhs - rhs).max() <= 1e-10 * np.abs(lhs).max()


def test_multigrid_cuts_iterations(mtn):
    """48 x 40 x 24 stretched mountain grid: flexible BiCGSTAB with the V-cycle
    reaches 1e-10 in at most a third of the iterations that the reference
    preconditioner needs."""
    from oracle.mg_oracle import Multigrid, apply, bicgstab, factors, pseudo_step
    cfg, coef = mtn
    f = cfg["fields"]
    b = cfg["rhs"]
    deta = 1.0 / (2 * (1 / f["dx"] ** 2 + 1 / f["dy"] ** 2))
    fac = factors(coef, deta)
    ref = lambda r: pseudo_step(coef, fac, deta, r, pseudo_step(coef, fac, deta, r, None))
    _, it_ref, res_ref = bicgstab(coef, ref, b)
    mg = Multigrid(coef, F.fcscal(cfg["dom"], f), f["dx"], f["dy"], dtau=2.0)
    x, it_mg, res_mg = bicgstab(coef, mg.cycle, b)
    assert res_ref <= 1e-10 and res_mg <= 1e-10
    assert 3 * it_mg <= it_ref, (it_mg, it_ref)
    r = b - apply(coef, x)
    assert np.sqrt(np.mean(r ** 2)) / np.sqrt(np.mean(b ** 2)) <= 1e-9


def test_bf16_rounding_is_round_to_nearest_even():
    """The oracle's BF16 rounding (of the FP32 rounding) against torch's
    float32 -> bfloat16 conversion, and on hand-picked ties."""
    import torch
    from oracle.mg_oracle import bf16
    rng = np.random.default_rng(0)
    x = rng.standard_normal(50000) * np.exp(rng.uniform(-40, 40, 50000))
    want = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(bf16(x), want)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to the even mantissa, 1
    ties = np.array([1 + 2.0 ** -8, 1 + 3 * 2.0 ** -8, -(1 + 2.0 ** -8)])
    assert np.array_equal(bf16(ties), [1.0, 1 + 2.0 ** -6, -1.0])


def test_vcycle_bf16_planes_differ_only_by_rounding(mtn):
    """With BF16 stencil planes the V-cycle moves by about the BF16 rounding
    (2^-9 relative), not more."""
    from oracle.mg_oracle import Multigrid
    cfg, coef = mtn
    f = cfg["fields"]
    b = np.random.default_rng(3).standard_normal(cfg["dom"].interior_shape)
    kw = dict(dtau=2.5)
    e32 = Multigrid(coef, F.fcscal(cfg["dom"], f), f["dx"], f["dy"], **kw).cycle(b)
    m16 = Multigrid(coef, F.fcscal(cfg["dom"], f), f["dx"], f["dy"], bf16_planes=True, **kw)
    e16 = m16.cycle(b)
    assert m16.levels[0]["scoef"] is not m16.levels[0]["coef"]
    assert m16.levels[-1]["scoef"] is m16.levels[-1]["coef"]
    rel = np.linalg.norm(e16 - e32) / np.linalg.norm(e32)
    assert 1e-6 < rel < 5e-2, rel


def test_e4m3_rounding_known_values():
    """The oracle's FP8 E4M3 rounding (the GPU's mg_smoother_fp8 copy) on the
    format's known values: normals, the largest finite value (saturation),
    subnormals (step 2^-9) and ties to even."""
    from oracle.mg_oracle import e4m3
    cases = [(1.0, 1.0), (-1.0, -1.0), (1.0625, 1.0), (1.1875, 1.25), (0.0625, 0.0625), (448.0, 448.0),
             (1000.0, 448.0), (2.0 ** -9, 2.0 ** -9), (2.0 ** -10, 0.0), (3 * 2.0 ** -10, 2.0 ** -8),
             (2.0 ** -6, 2.0 ** -6), (7 * 2.0 ** -9, 7 * 2.0 ** -9), (240.0, 240.0), (250.0, 256.0), (0.0, 0.0)]
    got = e4m3(np.array([c[0] for c in cases]))
    assert np.array_equal(got, np.array([c[1] for c in cases])), list(zip(cases, got))


def test_fp8_planes_scale_each_plane_to_the_top_binades():
    """Each plane's largest value lands in [64, 128) before rounding, so the
    FP8 copy keeps 3 bits of every value within 2^-6 of the plane's maximum
    and flushes values below 2^-16 of it."""
    from oracle.mg_oracle import fp8_planes
    rng = np.random.default_rng(3)
    planes = rng.standard_normal((3, 4, 5, 6)) * np.array([1e-6, 1.0, 3e4])[:, None, None, None]
    out = fp8_planes(planes)
    for p in range(3):
        big = np.abs(planes[p]) > np.abs(planes[p]).max() * 2.0 ** -6
        assert np.all(np.abs(out[p][big] - planes[p][big]) <= 2.0 ** -4 * np.abs(planes[p][big]))
    tiny = np.zeros((1, 2, 2, 2))
    tiny[0, 0, 0, 0] = 1.0
    tiny[0, 1, 1, 1] = 2.0 ** -18
    assert fp8_planes(tiny)[0, 1, 1, 1] == 0.0
