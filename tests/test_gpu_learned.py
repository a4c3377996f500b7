"""GPU: the learned network (fused forward, gradients, training) and what it
gains as a warm start and as a preconditioner stage.

Forward outputs (the fused cooperative kernel) and gradients (the training
path) are compared with the CPU oracle of the network (oracle/net_oracle.py)
evaluated with the same BF16 roundings; remaining differences come from FP32
accumulation order and rare BF16 rounding flips, so the tolerance is
norm-wise: 1e-2 for the forward output, 2e-2 per parameter block for the
gradients.

The gain tests pin the measured effect of training on small problems of the
training configuration (32 x 32 x 64): a regression of the trained network or
of the solver's use of it fails them.
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def netmod():
    from oracle import net_oracle as NO
    from pincflow_poisson import learned
    return learned, NO


def _random_params(NO, seed):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in NO.SIZES:
        if len(shape) > 1:
            d[name] = rng.uniform(-1, 1, shape) * np.sqrt(6.0 / shape[-1])
        else:
            d[name] = 0.1 * rng.standard_normal(shape)
    return NO.pack(d).astype(np.float32)


def _normwise(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_parameter_count(netmod):
    learned, NO = netmod
    assert NO.NPARAM == learned.NPARAM == 172_736


# grids with partial tiles (x not a multiple of 16, y not of 8), y_size 1,
# more tiles than SMs, and nz above and below the 64 levels of a column
@pytest.mark.parametrize("shape", [(64, 10, 12), (40, 9, 7), (96, 6, 8), (48, 1, 20), (32, 64, 160)])
def test_fused_forward_matches_oracle(shape, netmod):
    learned, NO = netmod
    p = _random_params(NO, 1)
    b = np.random.default_rng(2).standard_normal(shape)
    with learned.LearnedNet(max_columns=16384) as net:
        net.set_params(p)
        assert np.array_equal(net.get_params(), p)
        got = net.forward(b)
        again = net.forward(b)
    ref, _ = NO.forward(p.astype(np.float64), b, bf=True)
    assert np.array_equal(got, again)  # deterministic
    assert _normwise(got, ref) < 1e-2
    assert np.abs(got - ref).max() < 3e-2 * np.abs(ref).max()


def test_new_network_outputs_zero(netmod):
    learned, _ = netmod
    b = np.random.default_rng(3).standard_normal((64, 16, 16))
    with learned.LearnedNet(max_columns=256, seed=4) as net:
        assert not net.forward(b).any()


@pytest.mark.parametrize("shape", [(64, 12, 16), (48, 8, 8)])
def test_gradients_match_oracle(shape, netmod):
    learned, NO = netmod
    p = _random_params(NO, 3)
    rng = np.random.default_rng(4)
    b = rng.standard_normal(shape)
    x = rng.standard_normal(shape)
    with learned.LearnedNet(max_columns=4096) as net:
        net.set_params(p)
        loss, g = net.gradients(b, x)
    lref, gref = NO.loss_and_grad(p.astype(np.float64), b, x, bf=True)
    assert abs(loss - lref) <= 1e-3 * lref
    G, R = NO.unpack(g), NO.unpack(gref)
    for name, _ in NO.SIZES:
        assert _normwise(G[name], R[name]) < 2e-2, name


def test_save_load_roundtrip(netmod):
    learned, NO = netmod
    p = _random_params(NO, 5)
    with learned.LearnedNet(max_columns=64) as a, learned.LearnedNet(max_columns=64, seed=9) as b:
        a.set_params(p)
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "w.bin")
            a.save(path)
            b.load(path)
        assert np.array_equal(b.get_params(), p)


def test_bias_free_network_is_positively_homogeneous(netmod):
    learned, NO = netmod
    p = _random_params(NO, 6)
    b = np.random.default_rng(7).standard_normal((64, 8, 8))
    with learned.LearnedNet(max_columns=64) as net:
        net.set_params(p)
        net.set_bias_free(True)
        q = NO.unpack(net.get_params())
        assert not any(q[k].any() for k in NO.BIASES)
        y1, y2 = net.forward(b), net.forward(3.0 * b)
    assert _normwise(y2, 3.0 * y1) < 1e-2


def _solver(pcf, cfg):
    s = pcf.PoissonSolver(cfg["dom"], cfg["model"])
    s.set_grid(cfg["fields"])
    s.set_background(cfg["fields"])
    s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
    return s


def test_training_reduces_loss_and_warm_start_gains(netmod):
    """Trained on 24 plain-solver pairs of the training configuration, the warm
    start x0 = RMS(b) N(b / RMS(b)) approximates held-out solutions s* only
    loosely (relative error 0.74-0.86 measured, below 0.95 required; 1 for
    the untrained network), its initial FP64 true residual RMS(b - A x0) /
    RMS(b) is above 1 (measured 1.5-1.8: the network's error is rich in the
    short modes that A amplifies), and the mixed solves that start from it
    take the same iterations within +-4 (measured 52-56 against 53-55).  This
    pins the measured no-gain of the warm start."""
    learned, _ = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    pairs = learned.training_pairs(range(24), nx=32, ny=32, nz=64)
    assert len(pairs) == 24
    with learned.LearnedNet(max_columns=32 * 32, seed=1) as net:
        losses = learned.train(net, pairs, epochs=30, lr=2e-3)
        assert abs(losses[0] - 1.0) < 1e-6  # the untrained network outputs zero
        first, last = np.mean(losses[:24]), np.mean(losses[-24:])
        print(f"warm-start loss: first epoch {first:.4f}, last epoch {last:.4f}")
        assert last < 0.3, (first, last)
        ratios, errors, counts = [], [], []
        for i in range(100, 104):
            cfg = C.c3(i, nx=32, ny=32, nz=64)
            with _solver(pcf, cfg) as s:
                s.attach_network(net)
                kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed")
                sol, off = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(**kw))
                _, on = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(learned=True, **kw))
                assert not off.errflag and not on.errflag
                assert on.true_residual <= 1e-10
                # the solver's warm start x0 = RMS(b) N(b / RMS(b)), its error and FP64 true residual
                rms = np.sqrt(np.mean(cfg["rhs"] ** 2))
                x0 = rms * net.forward(cfg["rhs"] / rms)
                r0 = cfg["rhs"] - s.apply_operator(x0)
                ratios.append(float(np.sqrt(np.mean(r0 ** 2)) / rms))
                errors.append(float(np.linalg.norm(x0 - sol) / np.linalg.norm(sol)))
                counts.append((off.niter, on.niter))
        print("warm start: solution error", errors, "initial true residual", ratios, "iterations without / with",
              counts)
        assert max(errors) < 0.95, errors
        assert all(1.0 < r < 2.5 for r in ratios), ratios
        assert all(abs(b - a) <= 4 for a, b in counts), counts


def test_learned_preconditioner_stage(netmod):
    """The bias-free network trained on the multigrid V-cycle's (residual,
    error) pairs as a stage of the flexible FP32 BiCGSTAB's right
    preconditioner, z = M(r) + N(r - A M(r)): every solve reaches the FP64
    true residual 1e-10, none takes more iterations than the multigrid alone,
    and together they take at least 10 % fewer (measured 44 -> 35 on these
    four held-out problems)."""
    learned, _ = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    pairs = learned.preconditioner_pairs(range(24), nx=32, ny=32, nz=64)
    assert len(pairs) == 24
    with learned.LearnedNet(max_columns=32 * 32, seed=2) as net:
        net.set_bias_free(True)
        losses = learned.train(net, pairs, epochs=30, lr=2e-3)
        first, last = np.mean(losses[:24]), np.mean(losses[-24:])
        print(f"stage loss: first epoch {first:.4f}, last epoch {last:.4f}")
        assert last < first
        counts = []
        for i in range(100, 104):
            cfg = C.c3(i, nx=32, ny=32, nz=64)
            with _solver(pcf, cfg) as s:
                s.attach_network(net)
                kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed",
                          multigrid=True)
                _, off = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(**kw))
                x, on = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(learned=2, **kw))
                assert not off.errflag and not on.errflag, (off, on)
                assert on.true_residual <= 1e-10
                r = cfg["rhs"] - s.apply_operator(x)
                assert np.sqrt(np.mean(r ** 2)) / np.sqrt(np.mean(cfg["rhs"] ** 2)) <= 1.5e-10
                counts.append((off.niter, on.niter))
        print("multigrid iterations without / with the learned stage:", counts)
        assert all(b <= a for a, b in counts), counts
        assert sum(b for _, b in counts) <= 0.9 * sum(a for a, _ in counts), counts


def test_diverging_stage_falls_back_to_the_preconditioner(netmod):
    """A stage network with large random weights makes the flexible iteration
    diverge; the solve drops the stage, continues with the multigrid
    preconditioner alone from the last FP64 refinement, and still reaches
    1e-10."""
    learned, NO = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    p = _random_params(NO, 11) * 4.0
    cfg = C.c3(100, nx=32, ny=32, nz=64)
    with learned.LearnedNet(max_columns=32 * 32) as net, _solver(pcf, cfg) as s:
        net.set_params(p)
        net.set_bias_free(True)
        s.attach_network(net)
        kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed",
                  multigrid=True)
        x, on = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(learned=2, **kw))
        assert not on.errflag and on.true_residual <= 1e-10, on
        r = cfg["rhs"] - s.apply_operator(x)
        assert np.sqrt(np.mean(r ** 2)) / np.sqrt(np.mean(cfg["rhs"] ** 2)) <= 1.5e-10


@pytest.mark.parametrize("scale", [0.25, 1.0])
def test_unhelpful_stage_costs_a_bounded_number_of_iterations(netmod, scale):
    """Whatever the stage network does -- diverge, stall or merely not help --
    the mixed solve drops it after at most 60 iterations without convergence
    and finishes with the multigrid alone: it reaches 1e-10 in at most the
    multigrid's own count plus those 60 (and 8 of rounding slack)."""
    learned, NO = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    p = _random_params(NO, 12) * scale
    cfg = C.c3(101, nx=32, ny=32, nz=64)
    with learned.LearnedNet(max_columns=32 * 32) as net, _solver(pcf, cfg) as s:
        net.set_params(p)
        net.set_bias_free(True)
        s.attach_network(net)
        kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed",
                  multigrid=True)
        _, off = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(**kw))
        _, on = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(learned=2, **kw))
    assert not on.errflag and on.true_residual <= 1e-10, on
    assert on.niter <= off.niter + 60 + 8, (on.niter, off.niter)
