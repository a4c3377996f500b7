"""Learned warm start and preconditioner stage for the Poisson solve (no
reference counterpart).

The network (pcf_net in include/pincflow_poisson.h) works column by column:
a full 3x3 horizontal convolution of the input columns (resampled to 64
levels), a per-column MLP 64 -> 256 -> 256 -> 64, and a residual 3x3
convolution of its output; 172,736 parameters, BF16 weights, FP32
accumulation on the tensor cores.  It is trained on the GPU by the
library's own forward, backward and Adam kernels (pcf_net_train), on pairs
that the plain FP64 solver itself produces on the training configuration
(random Gaussian-hill terrain, 128 x 128 x 64; pincflow_poisson.configs.c3):
  * warm start: (right-hand side b, solution s) pairs; attached to a solver
    (PoissonSolver.attach_network) it provides the initial guess of the
    mixed-precision solve when PoissonNamelist.learned has bit 1;
  * preconditioner stage: bias-free, on the multigrid V-cycle's (residual,
    error) pairs; with bit 2 each preconditioner application of the flexible
    FP32 BiCGSTAB becomes z = M(r) + N(r - A M(r)).
The FP64 true residual still decides convergence.  No PyTorch: data sets go
to the device through the library.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from . import configs as C
from .solver import PoissonNamelist, PoissonSolver

NPARAM = 172_736


def _bind(lib):
    if getattr(lib, "_net_bound", False):
        return lib
    P = ctypes.POINTER
    vp, dp, fp = ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_float)
    lib.pcf_net_num_params.restype = ctypes.c_int
    lib.pcf_net_create.argtypes = [P(vp), ctypes.c_int, ctypes.c_longlong, ctypes.c_uint]
    lib.pcf_net_destroy.argtypes = [vp]
    lib.pcf_net_get_params.argtypes = [vp, fp]
    lib.pcf_net_set_params.argtypes = [vp, fp]
    lib.pcf_net_save.argtypes = [vp, ctypes.c_char_p]
    lib.pcf_net_load.argtypes = [vp, ctypes.c_char_p]
    lib.pcf_net_forward.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    lib.pcf_net_train_step.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       dp, fp]
    lib.pcf_net_gradients.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, fp]
    lib.pcf_net_train.argtypes = [vp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_uint, dp]
    lib.pcf_net_apply_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, vp, ctypes.c_int, vp]
    lib.pcf_set_network.argtypes = [vp, vp]
    lib.pcf_net_set_bias_free.argtypes = [vp, ctypes.c_int]
    for name in ("pcf_net_create", "pcf_net_destroy", "pcf_net_get_params", "pcf_net_set_params", "pcf_net_save",
                 "pcf_net_load", "pcf_net_forward", "pcf_net_train_step", "pcf_net_gradients", "pcf_set_network",
                 "pcf_net_set_bias_free", "pcf_net_train", "pcf_net_apply_device"):
        getattr(lib, name).restype = ctypes.c_int
    lib._net_bound = True
    return lib


class LearnedNet:
    """Owns one pcf_net on a device."""

    def __init__(self, device: int = 0, max_columns: int = 512 * 512, seed: int = 0):
        self.lib = _bind(_lib.load())
        assert self.lib.pcf_net_num_params() == NPARAM
        self._h = ctypes.c_void_p()
        _lib.check(self.lib.pcf_net_create(ctypes.byref(self._h), device, max_columns, seed), "pcf_net_create")

    def close(self):
        if self._h:
            self.lib.pcf_net_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_params(self) -> np.ndarray:
        p = np.zeros(NPARAM, dtype=np.float32)
        _lib.check(self.lib.pcf_net_get_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                   "pcf_net_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAM
        _lib.check(self.lib.pcf_net_set_params(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                   "pcf_net_set_params")

    def save(self, path: str):
        _lib.check(self.lib.pcf_net_save(self._h, path.encode()), "pcf_net_save")

    def load(self, path: str):
        _lib.check(self.lib.pcf_net_load(self._h, path.encode()), "pcf_net_load")

    def set_bias_free(self, on: bool = True):
        """Hold the biases at zero: N(a x) = a N(x) for a > 0 (the preconditioner stage)."""
        _lib.check(self.lib.pcf_net_set_bias_free(self._h, int(bool(on))), "pcf_net_set_bias_free")

    def forward(self, field: np.ndarray) -> np.ndarray:
        """N(field) for a host array of shape (nz, ny, nx)."""
        f = np.ascontiguousarray(field, dtype=np.float64)
        nz, ny, nx = f.shape
        out = np.zeros_like(f)
        _lib.check(self.lib.pcf_net_forward(self._h, _lib.dptr(f), nx, ny, nz, _lib.dptr(out)), "pcf_net_forward")
        return out

    def apply_device(self, d_in: int, d_out: int, shape, fp64: bool = False, scale_in: float = 1.0,
                     scale_out: float = 1.0, beta: float = 0.0, stream: int | None = None):
        """out = beta * out + scale_out * N(scale_in * in) on device fields (raw
        pointers, nz x ny x nx, FP64 or FP32), asynchronously on `stream` (a
        cudaStream_t as an integer; None: the network's own stream)."""
        nz, ny, nx = shape
        _lib.check(self.lib.pcf_net_apply_device(self._h, ctypes.c_void_p(d_in), nx, ny, nz, scale_in, scale_out,
                                                 beta, ctypes.c_void_p(d_out), int(bool(fp64)),
                                                 ctypes.c_void_p(stream) if stream else None),
                   "pcf_net_apply_device")

    def gradients(self, b: np.ndarray, x: np.ndarray):
        """(loss, gradient vector) for one sample, host arrays (nz, ny, nx)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        nz, ny, nx = b.shape
        loss = ctypes.c_double()
        g = np.zeros(NPARAM, dtype=np.float32)
        _lib.check(self.lib.pcf_net_gradients(self._h, _lib.dptr(b), _lib.dptr(x), nx, ny, nz, ctypes.byref(loss),
                                              g.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "pcf_net_gradients")
        return loss.value, g

    def train_step(self, d_b: int, d_x: int, shape, lr: float) -> float:
        """One Adam step on device FP32 fields (raw pointers), returns the loss."""
        nz, ny, nx = shape
        loss = ctypes.c_double()
        _lib.check(self.lib.pcf_net_train_step(self._h, ctypes.c_void_p(d_b), ctypes.c_void_p(d_x), nx, ny, nz, lr,
                                               ctypes.byref(loss), None), "pcf_net_train_step")
        return loss.value


def attach(solver: PoissonSolver, net: LearnedNet | None):
    lib = _bind(_lib.load())
    _lib.check(lib.pcf_set_network(solver._h, net.handle if net else None), "pcf_set_network")
    solver._net = net


def _problem(family, i, nx, ny, nz):
    """Training problem i: configs.c3 (the training configuration) or, with
    family "c5", a patch of the c5 family at c5's resolution (nx = ny)."""
    if family == "c5":
        return C.c5_patch(int(i), n=nx)
    return C.c3(int(i), nx=nx, ny=ny, nz=nz)


def training_pairs(indices, nx=128, ny=128, nz=64, tolerance=1e-8, device=0, family="c3"):
    """(b / RMS(b), s / RMS(b)) FP32 pairs from plain FP64 solves of the training
    configuration (configs.c3 with seeds `indices`, or c5 patches)."""
    out = []
    solver = None
    for i in indices:
        cfg = _problem(family, i, nx, ny, nz)
        if solver is None:
            solver = PoissonSolver(cfg["dom"], cfg["model"], device=device)
        solver.set_grid(cfg["fields"])
        solver.set_background(cfg["fields"])
        solver.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
        nl = PoissonNamelist(tolerance=tolerance, tolerance_is_relative=True, poisson_iterations=5000)
        s, info = solver.apply_bicgstab(cfg["rhs"], 1.0, nl)
        if info.errflag:
            continue
        rms = float(np.sqrt(np.mean(cfg["rhs"] ** 2)))
        out.append(((cfg["rhs"] / rms).astype(np.float32), (s / rms).astype(np.float32)))
    if solver is not None:
        solver.close()
    return out


def preconditioner_pairs(indices, nx=128, ny=128, nz=64, tolerance=1e-8, device=0, family="c3", **mg):
    """(r2 / RMS(r2), e / RMS(r2)) FP32 pairs for the learned preconditioner
    stage: for a training right-hand side b with plain FP64 solution s*, the
    multigrid V-cycle's output z = M(b) leaves the residual r2 = b - A z and
    the error e = s* - z, which the stage N(r2) should approximate.  The
    V-cycle is the solver's default one (BF16 operator copies on the two
    finest levels), as in the stage's solves; mg overrides its settings."""
    out = []
    solver = None
    nl_mg = PoissonNamelist(precision="mixed", multigrid=True, **mg)
    for i in indices:
        cfg = _problem(family, i, nx, ny, nz)
        if solver is None:
            solver = PoissonSolver(cfg["dom"], cfg["model"], device=device)
        solver.set_grid(cfg["fields"])
        solver.set_background(cfg["fields"])
        solver.compute_operator(cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], return_coef=False)
        nl = PoissonNamelist(tolerance=tolerance, tolerance_is_relative=True, poisson_iterations=5000)
        s, info = solver.apply_bicgstab(cfg["rhs"], 1.0, nl)
        if info.errflag:
            continue
        z = solver.apply_multigrid(cfg["rhs"], nl_mg)
        r2 = cfg["rhs"] - solver.apply_operator(z)
        e = s - z
        sc = float(np.sqrt(np.mean(r2 ** 2)))
        out.append(((r2 / sc).astype(np.float32), (e / sc).astype(np.float32)))
    if solver is not None:
        solver.close()
    return out


def train(net: LearnedNet, pairs, epochs: int = 4, lr: float = 1e-3, device: int = 0, log=None, seed: int = 0):
    """Adam over the pairs (one sample per step, `epochs` shuffled passes) on
    the device, through pcf_net_train.  Returns the per-step losses."""
    del device  # the network's own device
    b = np.ascontiguousarray(np.stack([p[0] for p in pairs]), dtype=np.float32)
    x = np.ascontiguousarray(np.stack([p[1] for p in pairs]), dtype=np.float32)
    count, nz, ny, nx = b.shape
    losses = np.zeros(count * epochs)
    t0 = time.time()
    fp = ctypes.POINTER(ctypes.c_float)
    _lib.check(net.lib.pcf_net_train(net.handle, b.ctypes.data_as(fp), x.ctypes.data_as(fp), count, nx, ny, nz,
                                     epochs, lr, seed, _lib.dptr(losses)), "pcf_net_train")
    if log:
        for ep in range(epochs):
            log(f"epoch {ep}: mean loss {np.mean(losses[ep * count:(ep + 1) * count]):.4f}")
        log(f"{count * epochs} steps in {time.time() - t0:.1f} s")
    return losses.tolist()


def evaluate(net: LearnedNet, indices, nx=128, ny=128, nz=64, device=0, **namelist):
    """Iterations and solve times with and without the learned warm start on
    configs.c3(index) problems: [(index, niter_without, niter_with, ms_without, ms_with)]."""
    out = []
    for i in indices:
        cfg = C.c3(int(i), nx=nx, ny=ny, nz=nz)
        with PoissonSolver(cfg["dom"], cfg["model"], device=device) as s:
            s.set_grid(cfg["fields"])
            s.set_background(cfg["fields"])
            dpip = np.zeros(cfg["dom"].halo_shape)
            args = (cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["tolref"])
            kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=5000, precision="mixed",
                      residual="true", **namelist)
            s.solve_poisson(*args, PoissonNamelist(**kw), dpip)  # warm-up (graph capture)
            a = s.solve_poisson(*args, PoissonNamelist(**kw), dpip)
            s.attach_network(net)
            s.solve_poisson(*args, PoissonNamelist(**kw, learned=True), dpip)
            b = s.solve_poisson(*args, PoissonNamelist(**kw, learned=True), dpip)
            s.attach_network(None)
        out.append((int(i), a.niter, b.niter, a.timings_ms["solve"], b.timings_ms["solve"]))
    return out


def evaluate_stage(net: LearnedNet, indices, nx=128, ny=128, nz=64, device=0):
    """Multigrid mixed solves with and without the learned preconditioner
    stage on configs.c3(index) problems:
    [(index, niter_without, niter_with, ms_without, ms_with)]."""
    out = []
    for i in indices:
        cfg = C.c3(int(i), nx=nx, ny=ny, nz=nz)
        with PoissonSolver(cfg["dom"], cfg["model"], device=device) as s:
            s.set_grid(cfg["fields"])
            s.set_background(cfg["fields"])
            dpip = np.zeros(cfg["dom"].halo_shape)
            args = (cfg["rhs"], cfg["rho"], cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], cfg["tolref"])
            kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=5000, precision="mixed",
                      residual="true", multigrid=True)
            s.solve_poisson(*args, PoissonNamelist(**kw), dpip)
            a = s.solve_poisson(*args, PoissonNamelist(**kw), dpip)
            s.attach_network(net)
            s.solve_poisson(*args, PoissonNamelist(**kw, learned=2), dpip)
            b = s.solve_poisson(*args, PoissonNamelist(**kw, learned=2), dpip)
            s.attach_network(None)
        out.append((int(i), a.niter, b.niter, a.timings_ms["solve"], b.timings_ms["solve"]))
    return out


def main(argv=None):
    """Training run of the learned part on the training configuration
    (configs.c3): generates the training pairs with the plain FP64 solver,
    trains with Adam on the GPU, evaluates on held-out problems, and writes
    the weights file.  --stage trains the bias-free preconditioner stage on
    the multigrid V-cycle's (residual, error) pairs instead of the warm
    start on (rhs, solution) pairs."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--pairs", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--size", default="128x128x64")
    ap.add_argument("--eval", type=int, default=8, help="held-out problems (configs.c3 indices from 100000)")
    ap.add_argument("--out", default=None, help="weights file to write")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--stage", action="store_true", help="train the preconditioner stage (bias-free)")
    ap.add_argument("--apply", type=int, default=0, metavar="N",
                    help="no training: apply a network with seeded random weights N times to a seeded random "
                         "field of --size (host arrays through pcf_net_forward; for profiling the fused kernel)")
    a = ap.parse_args(argv)
    nx, ny, nz = (int(v) for v in a.size.lower().split("x"))
    if a.apply:
        rng = np.random.default_rng(0)
        with LearnedNet(device=a.device, max_columns=nx * ny, seed=0) as net:
            p = net.get_params()
            p[:] = rng.uniform(-1, 1, p.size) * 0.05
            net.set_params(p)
            field = rng.standard_normal((nz, ny, nx))
            for _ in range(a.apply):
                out = net.forward(field)
        print(json.dumps({"applied": a.apply, "size": [nx, ny, nz], "mean_abs_out": float(np.abs(out).mean())}))
        return None
    t0 = time.time()
    make = preconditioner_pairs if a.stage else training_pairs
    pairs = make(range(a.pairs), nx=nx, ny=ny, nz=nz, device=a.device)
    t1 = time.time()
    net = LearnedNet(device=a.device, max_columns=nx * ny, seed=0)
    if a.stage:
        net.set_bias_free(True)
    losses = train(net, pairs, epochs=a.epochs, lr=a.lr, device=a.device,
                   log=lambda m: print(m, flush=True))
    t2 = time.time()
    if a.out:
        net.save(a.out)
    held = range(100000, 100000 + a.eval)
    summary = dict(role="preconditioner stage" if a.stage else "warm start", pairs=len(pairs), size=[nx, ny, nz],
                   generation_s=t1 - t0, training_s=t2 - t1, steps=len(losses),
                   loss_first_epoch=float(np.mean(losses[:len(pairs)])),
                   loss_last_epoch=float(np.mean(losses[-len(pairs):])))
    if a.stage:
        summary["stage_multigrid"] = evaluate_stage(net, held, nx, ny, nz, a.device)
    else:
        summary["warm_start_reference_preconditioner"] = evaluate(net, held, nx, ny, nz, a.device)
        summary["warm_start_multigrid"] = evaluate(net, held, nx, ny, nz, a.device, multigrid=True)
    print(json.dumps(summary), flush=True)
    net.close()
    return summary


if __name__ == "__main__":
    main()
