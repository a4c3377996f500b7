"""Benchmark: time to relative residual 1e-10 of the semi-implicit pressure
Poisson solve (PinCFlow.jl PoissonSolver) on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config c5|c2|c1|c4|step] [--method mg|mixed|fp64]

A step is one complete solve_poisson! (operator assembly, preconditioned
BiCGSTAB to FP64 true relative residual 1e-10, unscaling into dpip) of the
configuration's seeded synthetic workload.  The default workload is the
512 x 512 x 192 pseudo-incompressible domain (c5), whose 10 GB FP64 + 5 GB
FP32 operator is far larger than the 126 MB L2, so no flush is needed
between steps.  `value` is the device time per solve with inputs resident
in HBM (CUDA events on the solver's stream, max over ranks); `e2e` is the
host wall clock around the public host-array entry point, its
host<->device copies inside the timed region.  The same line carries the
learned arm (`learned`): the network trained on the training configuration
by the library's own kernels, used as warm start and as preconditioner
stage of the flexible FP32 BiCGSTAB, timed on the same inputs.

--impl reference times the reference algorithm on the host cores (the CPU
oracle, a C++ restatement of the Julia code; Julia is not available): the
operator assembly is timed once, and each step runs a bounded number of
BiCGSTAB iterations on the full workload, scaled to a complete solve by the
oracle's own iteration count for that workload.
--config step times the whole implicit half step around the solve
(implicit_integration!.jl:49-77: predictor, compute_lhs!, solve, correct!)
on the c2 grid, its roofline line the predictor kernels.
Multi-GPU runs are independent replicas (the solve does not shard across
GPUs in this build): weak scaling, one solve per rank per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "pincflow.jl_b200")
sys.path[:0] = [REPO, PKG]

import numpy as np  # noqa: E402

METRIC = "time to rel. residual 1e-10: learned+FP32-refined vs plain FP64 BiCGSTAB, 1 B200"
WORKLOADS = {
    "c2": "256x256x128 pseudo-incompressible, stretched terrain-following grid, Gaussian mountain 1 km, "
          "isothermal 250 K, RHS N(0,1) seed 12345",
    "c5": "512x512x192 pseudo-incompressible, 20 Gaussian ridges <= 2 km, wave-packet RHS",
    "c1": "periodic hill 40x1x40 Boussinesq, the 200 pressure solves of 100 time steps (rayleigh_factor 1, 2)",
    "c4": "32-member uneven ensemble, nx = ny in {64, 96, 128, 192}, nz = nx/2, random Gaussian hills and "
          "stratification, RHS N(0,1) per member",
    "step": "implicit half step (implicit_integration!.jl:49-77) on the c2 grid: implicit predictor, "
            "compute_lhs!, solve to 1e-10, correct!; winds and pi' N(0,1), rho' 1e-3 N(0,1) rhobar, seed 777",
}
STEP_METRIC = "time per implicit half step (predictor + compute_lhs! + solve to FP64 true rel. residual 1e-10 + " \
              "correct!), 1 B200"


DTYPES = {
    "mg": "f32+f64 (FP32 Krylov and preconditioner, FP64 true residual, refinement and dots; BF16 coefficient "
          "copies in the V-cycle's stencils on multigrid levels 0-1)",
    "mixed": "f32+f64 (FP32 Krylov and preconditioner, FP64 true residual, refinement and dots)",
    "fp64": "f64",
}

METHODS = {
    "mg": "flexible FP32 BiCGSTAB inside FP64 iterative refinement (reliable updates on the FP64 true residual), "
          "preconditioned by a horizontal aggregation multigrid V-cycle whose smoother is the reference "
          "line relaxation",
    "mixed": "flexible FP32 BiCGSTAB inside FP64 iterative refinement, reference preconditioner",
    "fp64": "plain FP64 BiCGSTAB, reference preconditioner",
}


def make_workload(name, seed_offset=0, size=None):
    from pincflow_poisson import configs
    if name == "c2":
        if size:
            nx, ny, nz = (int(v) for v in size.lower().split("x"))
            return configs.c2(seed=12345 + seed_offset, nx=nx, ny=ny, nz=nz)
        return configs.c2(seed=12345 + seed_offset)
    if name == "c5":
        return configs.c5(seed=5 + seed_offset)
    if name == "c1":
        return configs.c1(seed=seed_offset, step=0)
    raise SystemExit(f"unknown config {name}")


def step_state(cfg, seed):
    """Seeded predictands of the implicit-step workload (haloed arrays)."""
    dom = cfg["dom"]
    rng = np.random.default_rng(seed)
    u, v, w = (rng.standard_normal(dom.halo_shape) for _ in range(3))
    rhop = 1e-3 * rng.standard_normal(dom.halo_shape) * cfg["fields"]["rhobar"]
    pip = rng.standard_normal(dom.halo_shape)
    return dict(u=u, v=v, w=w, rho=np.ascontiguousarray(cfg["rho"]), rhop=rhop, pip=pip)


def oracle_step_parts(cfg, state):
    """Seconds of the oracle's predictor, compute_lhs! and corrector on the
    full workload (single-threaded loops), and the right-hand side."""
    from oracle import oracle as O
    O.build()
    dom, f = cfg["dom"], cfg["fields"]
    d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    model = O.MODELS[cfg["model"]]
    t0 = time.perf_counter()
    rho, rhop, u, v, w, pip, _, _ = O.implicit_predictor(d, model, f, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"],
                                                         state["rho"], state["rhop"], state["u"], state["v"],
                                                         state["w"], state["pip"])
    t1 = time.perf_counter()
    rhs, _ = O.compute_lhs(d, f, u, v, w, model=cfg["model"])
    t2 = time.perf_counter()
    O.correct(d, model, f, rho, cfg["betar"], cfg["dt"], cfg["rayleigh_factor"], np.zeros(dom.halo_shape), u, v, w,
              rhop, pip)
    t3 = time.perf_counter()
    return t1 - t0, t2 - t1, t3 - t2, rhs


def reference_step_seconds(cfg, state, sample_iters):
    """The oracle's implicit half step: predictor + compute_lhs! + assembly +
    `sample_iters` BiCGSTAB iterations scaled to the c2 oracle's full-solve
    iteration count + corrector.  Returns (seconds, threads, sample text)."""
    t_pred, t_lhs, t_corr, rhs = oracle_step_parts(cfg, state)
    c = dict(cfg)
    c["rhs"] = rhs
    niter, src = oracle_iterations("c2")
    t_asm, t_it, used = oracle_sample(c, sample_iters, os.cpu_count())
    total = t_pred + t_lhs + t_asm + t_it * (niter or 0) + t_corr
    sample = (f"oracle FP64 implicit predictor {t_pred:.2f} s, compute_lhs! {t_lhs:.2f} s and correct! {t_corr:.2f} s "
              f"(1 thread) + assembly {t_asm:.2f} s and {sample_iters} BiCGSTAB iterations on {used} threads scaled "
              f"to {niter} iterations ({src}, the c2 grid)")
    return total, used, sample


def max_over_ranks_of(x, device):
    """The maximum of x over the ranks of the default process group (x itself
    without one): every multi-GPU time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_bf16_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["bf16_tflops"])
    return 1590.0


def ncu_traffic(config, kernel="apply32"):
    """Per-launch DRAM bytes of a stencil family from the committed ncu summary, or None."""
    p = os.path.join(REPO, "profiles", f"stencil_{kernel}_{config}.txt")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        for line in fh:
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        under = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(under), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- CPU arm --

def oracle_sample(cfg, iters, threads=None):
    """Oracle FP64 assembly + `iters` BiCGSTAB iterations on the full workload.
    Returns (seconds_assembly, seconds_per_iteration, threads)."""
    smp = OracleSampler(cfg, threads)
    return smp.t_asm, smp.per_iteration(iters), smp.threads


# BiCGSTAB iterations per timed CPU sample: about 6 s of the 16 box cores on
# c2 (0.3 s per iteration) and 8 s on c5 (about 1.9 s per iteration)
SAMPLE_ITERS = {"c2": 20, "c5": 4, "step": 20}


def sample_iters(args):
    return args.ref_sample_iters or SAMPLE_ITERS.get(args.config, 3)


class OracleSampler:
    """The oracle's FP64 operator assembly of a workload, timed once, and
    bounded BiCGSTAB samples on that operator.  A sample of k iterations
    includes the solve's set-up (initial residual and norm, about an eighth
    of one iteration's work), so its per-iteration time is high by at most
    1/(8k)."""

    def __init__(self, cfg, threads=None):
        from oracle import oracle as O
        O.build()
        if threads:
            O.set_threads(threads)
        self.O, self.cfg = O, cfg
        dom, f = cfg["dom"], cfg["fields"]
        self.d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
        t0 = time.perf_counter()
        self.coef = O.compute_operator(self.d, O.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                                       cfg["rayleigh_factor"])
        self.t_asm = time.perf_counter() - t0
        self.threads = O.get_threads()

    def per_iteration(self, iters):
        f = self.cfg["fields"]
        t0 = time.perf_counter()
        _, info = self.O.bicgstab(self.d, self.coef, f["dx"], f["dy"], self.cfg["rhs"], tolerance=1e-30,
                                  tolerance_is_relative=True, poisson_iterations=iters)
        return (time.perf_counter() - t0) / max(info["niter"], 1)


def oracle_iterations(config):
    p = os.path.join(REPO, "tests", "golden", f"{config}_fp64_oracle.json")
    if os.path.exists(p):
        with open(p) as fh:
            return int(json.load(fh)["niter"]), "oracle full solve (tests/golden)"
    return None, None


def run_reference_c1(args, world):
    """The 200 periodic-hill solves on the oracle, on one thread: the reference
    runs single-threaded per MPI rank, and threads only add overhead to a
    1600-cell grid (measured 14.6 s on 16 threads against 3.0 s on one)."""
    from oracle import oracle as O
    from pincflow_poisson import configs as C
    O.build()
    O.set_threads(1)
    cfgs = [C.c1(seed=0, step=k) for k in range(200)]
    dom = cfgs[0]["dom"]
    d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for c in cfgs:
            O.solve_poisson(d, O.MODELS[c["model"]], c["fields"], c["rho"], c["betar"], c["rhs"], c["dt"],
                            c["rayleigh_factor"], tolerance=1e-10, tolerance_is_relative=True,
                            poisson_iterations=20000)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = statistics.mean(times)
    return value, "s", False, O.get_threads(), "per step: all 200 solves, oracle FP64 (assembly + BiCGSTAB)"


def run_reference_c4(args, world):
    """The 32 ensemble members on the oracle: assembly + a few iterations per
    size class, scaled by the oracle's full-solve iteration count of that
    class (tests/golden/c4_fp64_oracle.json) and summed over the members."""
    from pincflow_poisson import configs as C
    p = os.path.join(REPO, "tests", "golden", "c4_fp64_oracle.json")
    with open(p) as fh:
        counts = {int(k): v["niter"] for k, v in json.load(fh)["classes"].items()}
    sizes = C.c4_sizes()
    times = []
    for step in range(args.warmup + args.steps):
        per = {}
        for nx in sorted(set(sizes)):
            t_asm, t_it, used = oracle_sample(C.c4(sizes.index(nx), nx), sample_iters(args), os.cpu_count())
            per[nx] = t_asm + t_it * counts[nx]
        if step >= args.warmup:
            times.append(sum(per[nx] for nx in sizes))
    value = len(sizes) / statistics.mean(times)
    return value, "solves/s", True, used, (f"per step: oracle FP64 assembly + {sample_iters(args)} BiCGSTAB "
                                           "iterations per size class, scaled by the oracle's full-solve count "
                                           "of that class and summed over the 32 members")


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.config in ("c1", "c4", "step"):
        runner = {"c1": run_reference_c1, "c4": run_reference_c4, "step": run_reference_step}[args.config]
        value, unit, hib, used, sample = runner(args, world)
        metric = {"c1": "time for the 200 pressure solves of 100 steps to FP64 true rel. residual 1e-10, 1 B200",
                  "c4": "ensemble solves/s to FP64 true rel. residual 1e-10 (32 uneven members), 1 B200",
                  "step": STEP_METRIC}[args.config]
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": (value if unit == "s" else 32 / value) * 1e3,
                "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": f"{args.config}: {WORKLOADS[args.config]}",
                           "method": "plain FP64 BiCGSTAB with the reference preconditioner (CPU restatement "
                                     "of the Julia code)"},
                "cpu_baseline": {"value": value, "unit": unit, "cores": used, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    cfg = make_workload(args.config, size=args.size)
    niter, src = oracle_iterations(args.config)
    if niter is None:
        niter, src = args.ref_iterations, "--ref-iterations"
    k = sample_iters(args)
    smp = OracleSampler(cfg, os.cpu_count())  # the assembly, timed once
    per_it = []
    for step in range(args.warmup + args.steps):
        t_it = smp.per_iteration(k)
        if step >= args.warmup:
            per_it.append(t_it)
    t_it = statistics.mean(per_it)
    value = smp.t_asm + t_it * niter
    sample = (f"oracle FP64 operator assembly of the {args.config} workload timed once ({smp.t_asm:.2f} s), then "
              f"{k} BiCGSTAB iterations per step on {smp.threads} threads ({t_it:.3f} s per iteration over "
              f"{k * args.steps} timed iterations), scaled to {niter} iterations ({src})")
    line = {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.config}: {WORKLOADS[args.config]}", "method": "plain FP64 BiCGSTAB "
                       "with the reference preconditioner (CPU restatement of the Julia code)"},
            "seconds_per_iteration": t_it, "seconds_assembly": smp.t_asm, "iterations_scaled_to": niter,
            "cpu_baseline": {"value": value, "unit": "s", "cores": smp.threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------- implicit half step --

def run_step(args, rank, world, local_rank):
    """One step = implicit_integration!.jl:49-77 without output on device
    arrays: the implicit predictor with its boundary fills, compute_lhs!, the
    solve (--method) to FP64 true rel. residual 1e-10, the dpip fill and
    correct!.  Every step starts from the same seeded state (restored by a
    device copy outside the timed step)."""
    import torch

    import pincflow_poisson as pcf

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cfg = make_workload("c2", seed_offset=rank, size=args.size)
    dom, f = cfg["dom"], cfg["fields"]
    state = step_state(cfg, 777 + rank)
    s = pcf.PoissonSolver(dom, cfg["model"], device=local_rank)
    s.set_grid(f)
    s.set_background(f)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    pristine = {k: t(v) for k, v in state.items()}
    work = {k: v.clone() for k, v in pristine.items()}
    betar = t(cfg["betar"])
    dpip = torch.zeros(dom.halo_shape, dtype=torch.float64, device=dev)
    wold = torch.zeros(dom.halo_shape, dtype=torch.float64, device=dev)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000, residual="true")
    nl_fast = pcf.PoissonNamelist(**kw, precision="fp64" if args.method == "fp64" else "mixed",
                                  multigrid=args.method == "mg", mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse])
    nl_plain = pcf.PoissonNamelist(**kw, precision="fp64")

    def step(nl):
        for k in work:
            work[k].copy_(pristine[k])
        torch.cuda.synchronize()
        info = s.implicit_step_device(cfg["dt"], cfg["rayleigh_factor"], nl, *[work[k].data_ptr() for k in
                                      ("u", "v", "w", "rho", "rhop", "pip")], betar.data_ptr(), dpip.data_ptr(),
                                      d_wold=wold.data_ptr())
        if info.errflag:
            raise RuntimeError(f"step did not converge: {info}")
        return info

    for _ in range(args.warmup):
        step(nl_fast)
    l0 = s.launch_count
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        infos = [step(nl_fast) for _ in range(args.steps)]
        torch.cuda.synchronize()
    launches = s.launch_count - l0
    ms_per_step = max_over_ranks_of(statistics.mean(i.timings_ms["total"] for i in infos), dev)
    solve_ms = statistics.mean(i.timings_ms["solve"] + i.timings_ms["assemble"] for i in infos)

    s.profile(True)
    step(nl_fast)
    prof = s.profile_read()
    s.profile(False)
    plain = step(nl_plain)
    plain_s = max_over_ranks_of(plain.timings_ms["total"], dev) / 1e3

    # end to end: the host-array entry point with its copies, from pinned memory
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_betar = pin(cfg["betar"])
    e2e_s = []
    for _ in range(args.steps):
        h = {k: pin(v) for k, v in state.items()}
        h_dpip = pin(np.zeros(dom.halo_shape))
        t0 = time.perf_counter()
        info = s.implicit_step(cfg["dt"], cfg["rayleigh_factor"], nl_fast, h["u"], h["v"], h["w"], h["rho"],
                               h["rhop"], h["pip"], h_betar, h_dpip)
        e2e_s.append(time.perf_counter() - t0)
        if info.errflag:
            raise RuntimeError(f"e2e step did not converge: {info}")
    e2e = max_over_ranks_of(statistics.mean(e2e_s), dev)
    nh = int(np.prod(dom.halo_shape))
    if rank != 0:
        s.close()
        return
    peak, peak_kind = load_peaks()
    pr, co = prof["predict"], prof["correct"]
    pr_ms = pr["ms"] / max(pr["count"], 1)
    pr_bytes = pr["bytes"] / max(pr["count"], 1)
    achieved = pr_bytes / (pr_ms * 1e-3) / 1e9 if pr_ms > 0 else 0.0
    co_ms = co["ms"] / max(co["count"], 1)
    co_gbs = co["bytes"] / max(co["count"], 1) / (co_ms * 1e-3) / 1e9 if co_ms > 0 else None
    value = ms_per_step / 1e3
    line = {
        "metric": STEP_METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (predictor, corrector); solve " + DTYPES[args.method],
        "data": "synthetic",
        "config": {"workload": f"step: {WORKLOADS['step']}", "method": METHODS[args.method],
                   "l2": "fields of 73 MB each, ~20 of them per step: larger than L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "solve_ms_in_step": solve_ms, "iterations": infos[-1].niter,
        "plain_fp64_step_s": plain_s, "speedup_vs_plain_fp64_step": plain_s / value,
        "gpu_launches": launches,
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": 8 * 8 * nh, "d2h_bytes_per_step": 8 * 7 * nh},
        "roofline": {"bound": "hbm", "kernel": "implicit predictor: k_predict_uv, k_predict_w, k_predict_rhop and "
                     "two k_fill_predictands", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": pr_bytes, "ms_per_launch": pr_ms},
        "corrector": {"ms": co_ms, "gbs": co_gbs, "frac": co_gbs / peak if co_gbs else None},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        total, used, sample = reference_step_seconds(cfg, state, sample_iters(args))
        line["cpu_baseline"] = {"value": total, "unit": "s", "cores": used, "kind": "port", "sample": sample}
    print(json.dumps(line), flush=True)
    s.close()


def run_reference_step(args, world):
    cfg = make_workload("c2", size=args.size)
    state = step_state(cfg, 777)
    times = []
    for k in range(args.warmup + args.steps):
        total, used, sample = reference_step_seconds(cfg, state, sample_iters(args))
        if k >= args.warmup:
            times.append(total)
    return statistics.mean(times), "s", False, used, "per step: " + sample


# ------------------------------------------------------ periodic hill (c1) --

def run_c1(args, rank, world, local_rank):
    """C1: one step = the 200 pressure solves of 100 time steps of the periodic
    hill (2 per step, rayleigh_factor 1 and 2), each with its own seeded
    right-hand side, through one solver handle."""
    import torch

    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cfgs = [C.c1(seed=rank, step=k) for k in range(200)]
    dom, f = cfgs[0]["dom"], cfgs[0]["fields"]
    s = pcf.PoissonSolver(dom, cfgs[0]["model"], device=local_rank)
    s.set_grid(f)
    s.set_background(f)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ins = [(t(c["rhs"]), t(c["rho"]), t(c["betar"])) for c in cfgs]
    d_dpip = torch.zeros(dom.halo_shape, dtype=torch.float64, device=dev)
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000, residual="true")
    nl_fast = pcf.PoissonNamelist(**kw, precision="fp64" if args.method == "fp64" else "mixed",
                                  multigrid=args.method == "mg", mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse])
    nl_plain = pcf.PoissonNamelist(**kw, precision="fp64")

    def all_solves(nl):
        ms, it = 0.0, []
        for c, (r, rho, b) in zip(cfgs, ins):
            i = s.solve_poisson_device(r.data_ptr(), rho.data_ptr(), b.data_ptr(), c["dt"], c["rayleigh_factor"],
                                       c["tolref"], nl, d_dpip.data_ptr())
            if i.errflag:
                raise RuntimeError(f"solve did not converge: {i}")
            ms += i.timings_ms["total"]
            it.append(i.niter)
        return ms, it

    for _ in range(args.warmup):
        all_solves(nl_fast)
    torch.cuda.synchronize()
    l0 = s.launch_count
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        runs = [all_solves(nl_fast) for _ in range(args.steps)]
        wall = (time.perf_counter() - t0) / args.steps
    launches = s.launch_count - l0
    ms = statistics.mean(r[0] for r in runs)
    plain_ms, plain_it = all_solves(nl_plain)
    # end to end through the host-array entry point
    h = [(np.ascontiguousarray(c["rhs"]), np.ascontiguousarray(c["rho"]), np.ascontiguousarray(c["betar"]))
         for c in cfgs]
    hd = np.zeros(dom.halo_shape)
    t0 = time.perf_counter()
    for c, (r, rho, b) in zip(cfgs, h):
        s.solve_poisson(r, rho, b, c["dt"], c["rayleigh_factor"], c["tolref"], nl_fast, hd)
    e2e_s = time.perf_counter() - t0
    n = dom.nx * dom.ny * dom.nz
    if rank != 0:
        s.close()
        return
    line = {
        "metric": "time for the 200 pressure solves of 100 steps to FP64 true rel. residual 1e-10, 1 B200",
        "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (grids of at most 2048 cells take the single-block FP64 solver)", "data": "synthetic",
        "config": {"workload": f"c1: {WORKLOADS['c1']}", "method": METHODS[args.method],
                   "l2": "1600-cell grid: L2-resident by design (latency-bound workload)",
                   "parallelism": f"replicas x{world}"},
        "wall_s_per_step": wall, "plain_fp64_s": plain_ms / 1e3, "speedup_vs_plain_fp64": plain_ms / ms,
        "iterations_mean": statistics.mean(runs[-1][1]), "plain_fp64_iterations_mean": statistics.mean(plain_it),
        "solves_per_s": world * 200 / (ms / 1e3), "gpu_launches": launches,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 200 * 8 * (n + 2 * int(np.prod(dom.halo_shape))),
                "d2h_bytes_per_step": 200 * 8 * n},
        "roofline": {"bound": "latency", "note": "40x1x40 cells: each kernel moves a few tens of KB, so the solve "
                     "is bound by launch and dependency latency, not by HBM", "achieved": None, "peak": None,
                     "unit": "GB/s", "frac": None, "traffic": None},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        O.set_threads(1)
        d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
        t0 = time.perf_counter()
        for c in cfgs:
            O.solve_poisson(d, O.MODELS[c["model"]], c["fields"], c["rho"], c["betar"], c["rhs"], c["dt"],
                            c["rayleigh_factor"], tolerance=1e-10, tolerance_is_relative=True,
                            poisson_iterations=20000)
        line["cpu_baseline"] = {"value": time.perf_counter() - t0, "unit": "s", "cores": 1, "kind": "port",
                                "sample": "all 200 solves, oracle FP64 (assembly + BiCGSTAB), 1 thread"}
    print(json.dumps(line), flush=True)
    s.close()


# ---------------------------------------------------------- ensemble (c4) --

def run_ensemble(args, rank, world, local_rank):
    """C4: all members solved together (one graph launch per iteration batch
    for all members, tile shapes from the autotuner), against the same
    members solved one after another by the plain FP64 solver."""
    import torch

    import pincflow_poisson as pcf
    from pincflow_poisson import configs as C

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sizes = C.c4_sizes(seed=4 + rank)
    members = []
    for q, nx in enumerate(sizes):
        cfg = C.c4(1000 * rank + q, nx)
        s = pcf.PoissonSolver(cfg["dom"], cfg["model"], device=local_rank)
        s.set_grid(cfg["fields"])
        s.set_background(cfg["fields"])
        d = {k: torch.from_numpy(np.ascontiguousarray(cfg[k])).to(dev) for k in ("rhs", "rho", "betar")}
        d["dpip"] = torch.zeros(cfg["dom"].halo_shape, dtype=torch.float64, device=dev)
        members.append((cfg, s, d))
    torch.cuda.synchronize()
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000, residual="true")
    nl_ens = pcf.PoissonNamelist(**kw, precision="mixed", multigrid=True, mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse], autotune=True)
    nl_plain = pcf.PoissonNamelist(**kw, precision="fp64")
    ens = pcf.Ensemble([m[1] for m in members])
    cols = lambda key: [m[2][key].data_ptr() for m in members]
    scal = lambda key: [m[0][key] for m in members]

    def solve_all():
        infos = ens.solve_poisson_device(cols("rhs"), cols("rho"), cols("betar"), scal("dt"),
                                         scal("rayleigh_factor"), scal("tolref"), nl_ens, cols("dpip"))
        bad = [q for q, i in enumerate(infos) if i.errflag]
        if bad:
            raise RuntimeError(f"members {bad} did not converge")
        return infos

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return max_over_ranks_of(x, dev)

    for _ in range(args.warmup):
        solve_all()
    barrier()
    l0 = ens.launch_count
    with ClockSampler(local_rank) as clk:
        runs = [solve_all() for _ in range(args.steps)]
        barrier()
    launches = ens.launch_count - l0
    ms = max_over_ranks(statistics.mean(r[0].timings_ms["total"] for r in runs))
    n = len(members)
    value = world * n / (ms / 1e3)

    # the same members one after another: plain FP64, and the single-handle multigrid solve
    nl_single = pcf.PoissonNamelist(**kw, precision="mixed", multigrid=True, mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse], autotune=True)

    def sequential(nl):
        tot, iters = 0.0, []
        for cfg, s, d in members:
            i = s.solve_poisson_device(d["rhs"].data_ptr(), d["rho"].data_ptr(), d["betar"].data_ptr(), cfg["dt"],
                                       cfg["rayleigh_factor"], cfg["tolref"], nl, d["dpip"].data_ptr())
            if i.errflag:
                raise RuntimeError(f"sequential solve did not converge: {i}")
            tot += i.timings_ms["total"]
            iters.append(i.niter)
        return tot, iters

    sequential(nl_single)  # graphs captured for every member
    barrier()
    plain_ms, plain_iters = sequential(nl_plain)
    single_ms, single_iters = sequential(nl_single)
    plain_ms = max_over_ranks(plain_ms)
    single_ms = max_over_ranks(single_ms)

    # end to end: member inputs from pinned host memory, results back to the host
    hosts = [{k: torch.from_numpy(np.ascontiguousarray(m[0][k])).pin_memory() for k in ("rhs", "rho", "betar")}
             for m in members]
    outs = [torch.zeros(m[0]["dom"].halo_shape, dtype=torch.float64).pin_memory() for m in members]
    h2d = sum(int(h[k].numel()) * 8 for h in hosts for k in h)
    d2h = sum(int(o.numel()) * 8 for o in outs)
    barrier()
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for h, (_, _, d) in zip(hosts, members):
            for k in ("rhs", "rho", "betar"):
                d[k].copy_(h[k], non_blocking=True)
        torch.cuda.synchronize()
        solve_all()
        for o, (_, _, d) in zip(outs, members):
            o.copy_(d["dpip"], non_blocking=True)
        torch.cuda.synchronize()
        e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.mean(e2e))

    if rank != 0:
        ens.close()
        for m in members:
            m[1].close()
        return
    # roofline: the FP32 Krylov Total apply of the largest member, per-launch events
    big = max(range(n), key=lambda q: sizes[q])
    cfg, s, d = members[big]
    s.profile(True)
    s.solve_poisson_device(d["rhs"].data_ptr(), d["rho"].data_ptr(), d["betar"].data_ptr(), cfg["dt"],
                           cfg["rayleigh_factor"], cfg["tolref"], nl_single, d["dpip"].data_ptr())
    prof = s.profile_read()
    s.profile(False)
    a32 = prof["apply32"]
    kernel_ms = a32["ms"] / max(a32["count"], 1)
    bpl = a32["bytes"] / max(a32["count"], 1)
    peak, peak_kind = load_peaks()
    achieved = bpl / (kernel_ms * 1e-3) / 1e9 if kernel_ms > 0 else 0.0
    cells = sum(m[0]["dom"].nx * m[0]["dom"].ny * m[0]["dom"].nz for m in members)
    it = [i.niter for i in runs[-1]]
    line = {
        "metric": "ensemble solves/s to FP64 true rel. residual 1e-10 (32 uneven members), 1 B200",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPES["mg"],
        "data": "synthetic",
        "config": {"workload": f"c4: {WORKLOADS['c4']}", "members": sizes, "cells": cells,
                   "method": METHODS["mg"] + "; all members advanced together, one CUDA graph launch per "
                             "batch of iterations, stencil tiles from the autotuner",
                   "l2": "members total far above L2 (126 MB), no flush", "parallelism": f"replicas x{world}"},
        "iterations": it, "plain_fp64_iterations": plain_iters,
        "sequential_plain_fp64_solves_per_s": n / (plain_ms / 1e3),
        "sequential_single_mg_solves_per_s": n / (single_ms / 1e3),
        "speedup_vs_sequential_plain_fp64": plain_ms / ms,
        "speedup_vs_sequential_single_mg": single_ms / ms,
        "cell_updates_per_s": world * sum(m[0]["dom"].nx * m[0]["dom"].ny * m[0]["dom"].nz * 2 * i.niter
                                          for m, i in zip(members, runs[-1])) / (ms / 1e3),
        "gpu_launches": launches,
        "e2e": {"value": world * n / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "kernel": f"k_stencil Total apply FP32 of the {sizes[big]}^2 member",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": bpl,
                     "ms_per_launch": kernel_ms},
        "autotune": [{k: e[k] for k in ("kernel", "nx", "nz", "tile_x", "levels", "ms_best", "ms_default")}
                     for e in pcf.autotune_entries() if e["kernel"] == "total32_diff"],
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        # oracle assembly + 1 iteration per size class, scaled by each member's plain FP64 iteration count
        per_class = {}
        total = 0.0
        for (cfg, _, _), niter in zip(members, plain_iters):
            nx = cfg["dom"].nx
            if nx not in per_class:
                per_class[nx] = oracle_sample(cfg, 1, os.cpu_count())
            t_asm, t_it, used = per_class[nx]
            total += t_asm + t_it * niter
        line["cpu_baseline"] = {"value": n / total, "unit": "solves/s", "cores": used, "kind": "port",
                                "sample": "oracle FP64 assembly + 1 BiCGSTAB iteration per size class, scaled by "
                                          "each member's GPU FP64 iteration count and summed over the members"}
    print(json.dumps(line), flush=True)
    ens.close()
    for m in members:
        m[1].close()


# ----------------------------------------------------------------- GPU arm --

def deviation_vs_oracle(config, dpip):
    """Max pointwise deviation of the interior pressure `dpip` (nz, ny, nx)
    from the oracle's converged FP64 pressure of the same workload, at the
    cells of the committed fingerprint (tests/golden/<config>_fp64_fingerprint.npz,
    written by tests/golden/make_oracle_iterations.py): both solves leave the
    constant (null-space) component free, so the mean difference over the
    sampled cells is removed first; the deviation is relative to the largest
    |oracle - mean| there.  None without a fingerprint."""
    p = os.path.join(REPO, "tests", "golden", f"{config}_fp64_fingerprint.npz")
    if not os.path.exists(p):
        return None
    fp = np.load(p)
    if tuple(fp["shape"]) != tuple(dpip.shape):
        return None
    ref = fp["values"]
    got = dpip.ravel()[fp["indices"]]
    diff = got - ref
    dev = float(np.abs(diff - diff.mean()).max() / np.abs(ref - fp["mean"]).max())
    return {"value": dev, "cells": int(ref.size), "oracle_iterations": int(fp["niter"]),
            "oracle_true_residual": float(fp["true_residual"])}


def learned_arm(args, s, cfg, d_rhs, d_rho, d_betar, d_dpip, local_rank):
    """The learned part on this workload.  Two networks are trained on the
    training configuration (configs.c3 problems, 128 x 128 x 64 random
    Gaussian-hill terrain) by the library's own forward, backward and Adam
    kernels, on pairs that the plain FP64 solver generates:
      warm start: x0 = N(b), trained on (b, s) pairs;
      stage: each preconditioner application z = M(r) + N(r - A M(r)),
             bias-free, trained on the V-cycle's (residual, error) pairs.
    Each is then timed on this workload with the multigrid mixed solve to FP64
    true relative residual 1e-10 (data generation and training are set-up,
    reported, not timed)."""
    import pincflow_poisson as pcf
    from pincflow_poisson import learned as L
    dom = cfg["dom"]
    t0 = time.perf_counter()
    pairs = {"warm_start": L.training_pairs(range(args.learned_pairs), device=local_rank),
             "stage": L.preconditioner_pairs(range(args.learned_pairs), device=local_rank)}
    if args.config == "c5":
        # the same stage trained on 128 x 128 x 192 patches of the workload's own family
        pairs["stage_c5_patches"] = L.preconditioner_pairs(range(args.learned_pairs), nx=128, ny=128, nz=192,
                                                           device=local_rank, family="c5")
    t1 = time.perf_counter()
    cols = max(dom.nx * dom.ny, 128 * 128)
    nets, loss = {}, {}
    for q, role in enumerate(pairs):
        nets[role] = L.LearnedNet(device=local_rank, max_columns=cols, seed=q)
        if role != "warm_start":
            nets[role].set_bias_free(True)
        loss[role] = L.train(nets[role], pairs[role], epochs=args.learned_epochs, lr=args.learned_lr,
                             device=local_rank)
    t2 = time.perf_counter()
    kw = dict(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000, precision="mixed",
              residual="true", multigrid=args.method == "mg", mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse])
    out = {"training": {"configuration": "c3: 128x128x64 Boussinesq, 1-5 Gaussian hills, N ~ U(0.005, 0.02); "
                                         "stage_c5_patches: 128x128x192 patches of the c5 family at its resolution",
                        "pairs": {r: len(p) for r, p in pairs.items()}, "epochs": args.learned_epochs,
                        "lr": args.learned_lr,
                        "generation_s": t1 - t0, "training_s": t2 - t1, "parameters": L.NPARAM}}
    for role in nets:
        bit = 1 if role == "warm_start" else 2
        s.attach_network(nets[role])
        nl = pcf.PoissonNamelist(**kw, learned=bit)
        infos = []
        for k in range(1 + min(args.steps, 3)):  # the first solve captures the graphs
            i = s.solve_poisson_device(d_rhs.data_ptr(), d_rho.data_ptr(), d_betar.data_ptr(), cfg["dt"],
                                       cfg["rayleigh_factor"], cfg["tolref"], nl, d_dpip.data_ptr())
            if k:
                infos.append(i)
        s.attach_network(None)
        out[role] = {"s": statistics.mean(i.timings_ms["total"] for i in infos) / 1e3, "iterations": infos[-1].niter,
                     "true_residual": infos[-1].true_residual, "converged": not infos[-1].errflag,
                     "loss_first_epoch": float(np.mean(loss[role][:len(pairs[role])])),
                     "loss_last_epoch": float(np.mean(loss[role][-len(pairs[role]):]))}
    # the fused network kernel alone on this grid: CUDA events around
    # back-to-back applications on an FP32 field (the stage's case)
    import torch
    shape = (dom.nz, dom.ny, dom.nx)
    f_in = torch.randn(shape, dtype=torch.float32, device=d_rhs.device)
    f_out = torch.empty_like(f_in)
    st = torch.cuda.Stream(d_rhs.device)  # a stream of its own: a null handle would mean the network's stream
    net = nets["stage"]
    torch.cuda.synchronize()
    for _ in range(3):
        net.apply_device(f_in.data_ptr(), f_out.data_ptr(), shape, stream=st.cuda_stream)
    reps = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        net.apply_device(f_in.data_ptr(), f_out.data_ptr(), shape, stream=st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    cols = dom.nx * dom.ny
    flop = cols * 2.0 * (2 * 64 * 576 + 64 * 256 + 256 * 256 + 256 * 64)
    peak_tf = load_bf16_peak()
    out["network_kernel"] = {"kernel": "k_net_fused (gather, 3x3 convolution, MLP and output convolution in one "
                                       "cooperative tcgen05 kernel)", "columns": cols, "ms_per_application": ms,
                             "flop_per_application": flop, "tflops": flop / (ms * 1e-3) / 1e12,
                             "tensor_peak_tflops": peak_tf, "frac": flop / (ms * 1e-3) / 1e12 / peak_tf}
    for n in nets.values():
        n.close()
    return out



def run_ours(args, rank, world, local_rank):
    import torch

    import pincflow_poisson as pcf

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod

    cfg = make_workload(args.config, seed_offset=rank, size=args.size)
    dom, f = cfg["dom"], cfg["fields"]
    dev = torch.device("cuda", local_rank)
    s = pcf.PoissonSolver(dom, cfg["model"], device=local_rank)
    s.set_grid(f)
    s.set_background(f)

    def dev_tensor(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    d_rhs, d_rho, d_betar = dev_tensor(cfg["rhs"]), dev_tensor(cfg["rho"]), dev_tensor(cfg["betar"])
    d_dpip = torch.zeros(dom.halo_shape, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    nl_fast = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000,
                                  precision="fp64" if args.method == "fp64" else "mixed", residual="true",
                                  multigrid=args.method == "mg", mg_dtau=args.mg_dtau, mg_fused_coarse=FUSED[args.fused_coarse])
    nl_plain = pcf.PoissonNamelist(tolerance=1e-10, tolerance_is_relative=True, poisson_iterations=20000,
                                   precision="fp64", residual="true")

    def solve_dev(nl):
        info = s.solve_poisson_device(d_rhs.data_ptr(), d_rho.data_ptr(), d_betar.data_ptr(), cfg["dt"],
                                      cfg["rayleigh_factor"], cfg["tolref"], nl, d_dpip.data_ptr())
        if info.errflag:
            raise RuntimeError(f"solve did not converge: {info}")
        return info

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return max_over_ranks_of(x, dev)

    for _ in range(args.warmup):
        solve_dev(nl_fast)

    # --- headline: device-resident inputs (iteration batches replay as CUDA graphs)
    l0 = s.launch_count
    barrier()
    infos = []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            infos.append(solve_dev(nl_fast))
        barrier()
    launches = s.launch_count - l0
    ms = [i.timings_ms["total"] for i in infos]
    ms_per_step = max_over_ranks(statistics.mean(ms))
    value = ms_per_step / 1e3

    # --- per-kernel device times: the same steps again, each launch timed with
    # CUDA events on the solver's stream (direct launches, no graphs)
    s.profile(True)
    barrier()
    prof_infos = [solve_dev(nl_fast) for _ in range(args.steps)]
    barrier()
    prof = s.profile_read()
    s.profile(False)
    profiled_ms = statistics.mean(i.timings_ms["total"] for i in prof_infos)

    # --- plain FP64 BiCGSTAB on the same inputs ---------------------------
    fast_dpip = dom.interior(d_dpip.cpu().numpy()).copy()
    barrier()
    plain = [solve_dev(nl_plain) for _ in range(args.plain_steps)]
    barrier()
    plain_dpip = dom.interior(d_dpip.cpu().numpy()).copy()
    # both solves leave the constant (null-space) component of dpip free
    diff = fast_dpip - plain_dpip
    dev_max = float(np.abs(diff - diff.mean()).max() / np.abs(plain_dpip - plain_dpip.mean()).max())
    plain_s = max_over_ranks(statistics.mean(i.timings_ms["total"] for i in plain)) / 1e3
    dev_oracle = deviation_vs_oracle(args.config, fast_dpip) if rank == 0 and not args.size else None

    # --- the learned arm: warm start + preconditioner stage ---------------
    learned = None if args.no_learned else learned_arm(args, s, cfg, d_rhs, d_rho, d_betar, d_dpip, local_rank)

    # --- end to end through the host-array entry point --------------------
    h_rhs = torch.from_numpy(np.ascontiguousarray(cfg["rhs"])).pin_memory().numpy()
    h_rho = torch.from_numpy(np.ascontiguousarray(cfg["rho"])).pin_memory().numpy()
    h_betar = torch.from_numpy(np.ascontiguousarray(cfg["betar"])).pin_memory().numpy()
    h_dpip = torch.zeros(dom.halo_shape, dtype=torch.float64).pin_memory().numpy()
    barrier()
    e2e_ms, e2e_wall = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        info = s.solve_poisson(h_rhs, h_rho, h_betar, cfg["dt"], cfg["rayleigh_factor"], cfg["tolref"],
                               nl_fast, h_dpip)
        e2e_wall.append(time.perf_counter() - t0)
        if info.errflag:
            raise RuntimeError(f"e2e solve did not converge: {info}")
        e2e_ms.append(info.timings_ms["total"])
    barrier()
    e2e_s = max_over_ranks(statistics.mean(e2e_wall))
    n = dom.nx * dom.ny * dom.nz
    nh = int(np.prod(dom.halo_shape))
    h2d = 8 * (n + 2 * nh)
    d2h = 8 * n

    if rank != 0:
        s.close()
        return

    # --- roofline of the dominant kernel: the single-kernel family with the
    # largest share of the profiled solve ("mg" gathers many coarse-level
    # kernels and is not one kernel) ----------------------------------------
    peak, peak_kind = load_peaks()
    f32 = args.method != "fp64"
    names = {"apply32": "k_stencil Total apply FP32 (Krylov, difference form, fused dot)",
             "apply64": "k_stencil Total apply FP64", "pseudo32": "k_stencil Horizontal apply + pseudo-step FP32",
             "pseudo64": "k_stencil Horizontal apply + pseudo-step FP64",
             "thomas32": "k_thomas column solves FP32", "thomas64": "k_thomas column solves FP64",
             "mg_bf16": "k_stencil V-cycle finest-level residual / pseudo-step on the BF16 operator copy, "
                        "coefficient tiles staged in shared memory by TMA on grids 128 or more wide"}

    def roof(tag):
        v = prof[tag]
        k_ms = v["ms"] / max(v["count"], 1)
        b = v["bytes"] / max(v["count"], 1)
        ach = b / (k_ms * 1e-3) / 1e9 if k_ms > 0 else 0.0
        return {"bound": "hbm", "kernel": names[tag], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": ncu_traffic(args.config, tag),
                "algorithmic_bytes_per_launch": b, "ms_per_launch": k_ms}

    dominant = max((t for t in names if prof[t]["count"]), key=lambda t: prof[t]["ms"])
    krylov = "apply32" if f32 else "apply64"
    total_prof_ms = sum(v["ms"] for v in prof.values())
    shares = {k: round(v["ms"] / total_prof_ms, 4) for k, v in prof.items() if v["count"]} if total_prof_ms else {}
    per_kernel = {k: {"launches": v["count"], "ms_per_launch": v["ms"] / v["count"],
                      "gbs": v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] > 0 else None}
                  for k, v in prof.items() if v["count"]}

    last = infos[-1]
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPES[args.method], "data": "synthetic",
        "config": {"workload": f"{args.config}: {WORKLOADS[args.config]}",
                   "method": METHODS[args.method],
                   "convergence": "FP64 true residual RMS(b-Ax)/RMS(b) <= 1e-10",
                   "l2": f"inputs larger than L2 (operator {25 * n * 8 / 1e9:.1f} GB FP64 + "
                         f"{25 * n * 4 / 1e9:.1f} GB FP32 x 2 forms vs 126 MB L2), no flush",
                   "parallelism": f"replicas x{world}"},
        "plain_fp64_s": plain_s, "speedup_vs_plain_fp64": plain_s / value,
        "iterations": last.niter, "refinements": last.nrefine, "true_residual": last.true_residual,
        "plain_fp64_iterations": plain[-1].niter,
        "max_pointwise_dev_vs_plain_fp64": dev_max,
        "max_pointwise_dev_vs_oracle": dev_oracle,
        "solves_per_s": world / value,
        "cell_updates_per_s": world * n * (2 * last.niter) / value,
        "gpu_launches": launches,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "clock": "host wall clock around PoissonSolver.solve_poisson (pcf_solve) on pinned host arrays",
                "device_events_s": statistics.mean(e2e_ms) / 1e3},
        "roofline": roof(dominant),
        "roofline_krylov_apply": roof(krylov),
        "learned": learned,
        "kernel_shares": shares, "kernels": per_kernel,
        "kernel_timing": f"CUDA events around every launch of {args.steps} profiled solves run right after the "
                         f"timed region (direct launches; {profiled_ms:.1f} ms per solve)",
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        niter, src = oracle_iterations(args.config)
        if niter is None or args.size:
            niter, src = plain[-1].niter, "the GPU FP64 solve's iteration count"
        k = sample_iters(args)
        smp = OracleSampler(cfg, os.cpu_count())
        t_it = smp.per_iteration(k)
        line["cpu_baseline"] = {
            "value": smp.t_asm + t_it * niter, "unit": "s", "cores": smp.threads, "kind": "port",
            "sample": f"oracle FP64 assembly ({smp.t_asm:.2f} s) + {k} BiCGSTAB iterations of the same workload "
                      f"({t_it:.3f} s each), scaled to {niter} iterations ({src})"}
        del smp
    print(json.dumps(line), flush=True)
    s.close()


FUSED = {"auto": None, "on": True, "off": False}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=sorted(WORKLOADS))
    ap.add_argument("--size", default=None,
                    help="c2 and step only: NXxNYxNZ instead of 256x256x128 (profiling captures)")
    ap.add_argument("--method", default="mg", choices=sorted(METHODS))
    ap.add_argument("--mg-dtau", type=float, default=2.5)
    ap.add_argument("--fused-coarse", default="auto", choices=["auto", "on", "off"],
                    help="multigrid: the coarse levels as one cluster launch per cycle (mg_fused_coarse; auto: "
                         "in the ensemble only)")
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--ref-sample-iters", type=int, default=None,
                    help="BiCGSTAB iterations per CPU sample (default: 20 on c2 and step, 4 on c5, 3 on c4)")
    ap.add_argument("--ref-iterations", type=int, default=450)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned arm")
    ap.add_argument("--learned-pairs", type=int, default=48, help="training pairs of each network")
    ap.add_argument("--learned-epochs", type=int, default=16)
    ap.add_argument("--learned-lr", type=float, default=2e-3)
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.size and args.config not in ("c2", "step"):
        raise SystemExit("--size applies to --config c2 and step only")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.config == "c4":
            run_ensemble(args, rank, world, local_rank)
        elif args.config == "c1":
            run_c1(args, rank, world, local_rank)
        elif args.config == "step":
            run_step(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
