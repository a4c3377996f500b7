"""Runs the CPU oracle's FP64 BiCGSTAB (the reference algorithm) to relative
residual 1e-10 on a full benchmark workload and records
  * tests/golden/<config>_fp64_oracle.json: the iteration count, the final
    residual and the run time (bench.py scales its bounded CPU samples by
    these counts);
  * tests/golden/<config>_fp64_fingerprint.npz (c2, c5; c4_<nx>_... for the
    first member of each c4 size class): a fingerprint of
    the oracle's converged pressure dpip = solution / fcscal / dt
    (solve_poisson!.jl:65-72): its values at FINGERPRINT_POINTS seeded
    interior cells, its mean and the RMS of each z-level with the mean
    removed.  The solve leaves the constant (null-space) component of dpip
    free, so comparisons remove the offset first.  tests/test_gpu_baseline
    compares the GPU solve of the same workload with it.

  c2   the 256 x 256 x 128 pseudo-incompressible workload (about 15 min on 8 cores)
  c5   the 512 x 512 x 192 workload (about 100 min on 8 cores)
  c4   the first ensemble member of every size class (about 10 min on 8 cores)

Usage: python tests/golden/make_oracle_iterations.py c2|c5|c4
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "pincflow.jl_b200")]

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402
from pincflow_poisson import configs as C  # noqa: E402

FINGERPRINT_POINTS = 65536
FINGERPRINT_SEED = 20261203


def fingerprint_indices(n_cells):
    """Sorted distinct flat interior indices (x fastest) of the fingerprint."""
    rng = np.random.default_rng(FINGERPRINT_SEED)
    idx = np.unique(rng.integers(0, n_cells, size=2 * FINGERPRINT_POINTS))
    return rng.permutation(idx)[:FINGERPRINT_POINTS].astype(np.int64).copy()


def full_solve(cfg, label, fingerprint=None):
    dom, f = cfg["dom"], cfg["fields"]
    d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
    t0 = time.time()
    coef = O.compute_operator(d, O.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                              cfg["rayleigh_factor"])
    t1 = time.time()
    sol, info = O.bicgstab(d, coef, f["dx"], f["dy"], cfg["rhs"], tolerance=1e-10, tolerance_is_relative=True,
                           poisson_iterations=5000)
    t2 = time.time()
    r = cfg["rhs"] - O.apply_operator(d, coef, sol)
    true_res = float(np.sqrt((r ** 2).mean()) / np.sqrt((cfg["rhs"] ** 2).mean()))
    out = dict(workload=label, niter=info["niter"], errflag=info["errflag"], residual=float(info["residual"]),
               true_residual=true_res, seconds_assembly=t1 - t0, seconds_bicgstab=t2 - t1,
               threads=O.get_threads(), solution_rms=float(np.sqrt((sol ** 2).mean())),
               solution_checksum=float(np.abs(sol).sum()))
    if fingerprint:
        # solve_poisson!.jl:65-72: solution ./= sqrt(pbar^2 / rhobar); dpip = solution / dt
        pb, rb = dom.interior(f["pbar"]), dom.interior(f["rhobar"])
        dpip = sol / np.sqrt(pb * pb / rb) / cfg["dt"]
        mean = float(dpip.mean())
        idx = fingerprint_indices(dpip.size)
        level_rms = np.sqrt(((dpip - mean) ** 2).mean(axis=(1, 2)))
        np.savez_compressed(fingerprint, indices=idx, values=dpip.ravel()[idx], mean=mean, level_rms=level_rms,
                            shape=np.array(dpip.shape), niter=info["niter"], true_residual=true_res,
                            seed=FINGERPRINT_SEED)
        out["fingerprint"] = os.path.basename(fingerprint)
    return out


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "c2"
    fp = os.path.join(HERE, f"{which}_fp64_fingerprint.npz")
    if which == "c2":
        out = full_solve(C.c2(), "c2 256x256x128 PseudoIncompressible seed 12345", fp)
    elif which == "c5":
        out = full_solve(C.c5(), "c5 512x512x192 PseudoIncompressible seed 5", fp)
    elif which == "c4":
        sizes = C.c4_sizes()
        out = {"workload": "c4 ensemble (seed 4): first member of each size class", "classes": {}}
        for nx in sorted(set(sizes)):
            q = sizes.index(nx)
            fpq = os.path.join(HERE, f"c4_{nx}_fp64_fingerprint.npz")
            out["classes"][str(nx)] = dict(full_solve(C.c4(q, nx), f"c4 member {q}, {nx}x{nx}x{nx // 2}", fpq),
                                           member=q)
            print(nx, out["classes"][str(nx)], flush=True)
    else:
        raise SystemExit(f"unknown config {which}")
    with open(os.path.join(HERE, f"{which}_fp64_oracle.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
