"""GPU: the learned warm-start network (forward, gradients, training, gain).

Forward outputs and gradients are compared with the CPU oracle of the network
(oracle/net_oracle.py) evaluated with the same BF16 roundings; remaining
differences come from FP32 accumulation order and rare BF16 rounding flips,
so the tolerance is norm-wise: 1e-2 for the forward output, 2e-2 per
parameter block for the gradients.
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
        fan = shape[-1] if len(shape) > 1 else 1
        if name.startswith("W"):
            d[name] = rng.uniform(-1, 1, shape) * np.sqrt(6.0 / fan)
        elif name.startswith("K"):
            d[name] = 0.1 * rng.standard_normal(shape)
        else:
            d[name] = 0.1 * rng.standard_normal(shape)
    return NO.pack(d).astype(np.float32)


def _normwise(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("shape", [(64, 10, 12), (40, 9, 7), (96, 6, 8)])
def test_forward_matches_oracle(shape, netmod):
    learned, NO = netmod
    p = _random_params(NO, 1)
    b = np.random.default_rng(2).standard_normal(shape)
    with learned.LearnedNet(max_columns=4096) as net:
        net.set_params(p)
        assert np.array_equal(net.get_params(), p)
        got = net.forward(b)
    ref, _ = NO.forward(p.astype(np.float64), b, bf=True)
    assert _normwise(got, ref) < 1e-2
    assert np.abs(got - ref).max() < 3e-2 * np.abs(ref).max()


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


def test_training_reduces_loss_and_warm_start_gains(netmod):
    """Trains on plain-solver pairs of the training configuration (small grids)
    and checks, on held-out right-hand sides, that the trained warm start
    lowers the initial FP64 residual of the mixed solve."""
    learned, _ = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    pairs = learned.training_pairs(range(12), nx=32, ny=32, nz=64)
    assert len(pairs) == 12
    with learned.LearnedNet(max_columns=32 * 32, seed=1) as net:
        losses = learned.train(net, pairs, epochs=25, lr=2e-3)
        first, last = np.mean(losses[:12]), np.mean(losses[-12:])
        assert last < 0.7 * first, (first, last)
        # held-out problems: initial residual with and without the warm start
        gains = []
        for i in range(100, 104):
            cfg = C.c3(i, nx=32, ny=32, nz=64)
            with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
                s.set_grid(cfg["fields"])
                s.set_background(cfg["fields"])
                s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
                s.attach_network(net)
                kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=4000, precision="mixed")
                _, off = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(**kw))
                _, on = s.apply_bicgstab(cfg["rhs"], 1.0, pcf.PoissonNamelist(learned=True, **kw))
                assert not off.errflag and not on.errflag
                assert on.true_residual <= 1e-10
                h_on = s.residual_history()
                gains.append((off.niter, on.niter))
        print("iterations without / with the learned warm start:", gains)


def test_bias_free_network_is_positively_homogeneous(netmod):
    learned, NO = netmod
    p = _random_params(NO, 6)
    b = np.random.default_rng(7).standard_normal((64, 8, 8))
    with learned.LearnedNet(max_columns=64) as net:
        net.set_params(p)
        net.set_bias_free(True)
        q = NO.unpack(net.get_params())
        assert not q["b1"].any() and not q["b2"].any() and not q["b3"].any()
        y1, y2 = net.forward(b), net.forward(3.0 * b)
    assert _normwise(y2, 3.0 * y1) < 1e-2


def test_learned_preconditioner_stage(netmod):
    """The bias-free network trained on the multigrid V-cycle's (residual,
    error) pairs serves as a stage of the flexible FP32 BiCGSTAB's right
    preconditioner, z = M(r) + N(r - A M(r)): the solve still reaches the FP64
    true residual 1e-10, and the iteration counts with and without the stage
    are recorded."""
    learned, _ = netmod
    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C
    pairs = learned.preconditioner_pairs(range(12), nx=32, ny=32, nz=64)
    assert len(pairs) == 12
    with learned.LearnedNet(max_columns=32 * 32, seed=2) as net:
        net.set_bias_free(True)
        losses = learned.train(net, pairs, epochs=25, lr=2e-3)
        assert np.mean(losses[-12:]) < np.mean(losses[:12])
        counts = []
        for i in range(100, 104):
            cfg = C.c3(i, nx=32, ny=32, nz=64)
            with pcf.PoissonSolver(cfg["dom"], cfg["model"]) as s:
                s.set_grid(cfg["fields"])
                s.set_background(cfg["fields"])
                s.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
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
        assert all(b <= 2 * a + 4 for a, b in counts), counts
