"""Runs the CPU oracle's FP64 BiCGSTAB (the reference algorithm) to relative
residual 1e-10 on a full benchmark workload and records the iteration count,
the final residual and the run time in tests/golden/<config>_fp64_oracle.json.
bench.py scales its bounded CPU samples by these counts.

  c2   the 256 x 256 x 128 pseudo-incompressible workload (about 15 min on 8 cores)
  c5   the 512 x 512 x 192 workload (a few hours on 8 cores)
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


def full_solve(cfg, label):
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
    return dict(workload=label, niter=info["niter"], errflag=info["errflag"], residual=float(info["residual"]),
                true_residual=true_res, seconds_assembly=t1 - t0, seconds_bicgstab=t2 - t1,
                threads=O.get_threads(), solution_rms=float(np.sqrt((sol ** 2).mean())),
                solution_checksum=float(np.abs(sol).sum()))


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "c2"
    if which == "c2":
        out = full_solve(C.c2(), "c2 256x256x128 PseudoIncompressible seed 12345")
    elif which == "c5":
        out = full_solve(C.c5(), "c5 512x512x192 PseudoIncompressible seed 5")
    elif which == "c4":
        sizes = C.c4_sizes()
        out = {"workload": "c4 ensemble (seed 4): first member of each size class", "classes": {}}
        for nx in sorted(set(sizes)):
            q = sizes.index(nx)
            out["classes"][str(nx)] = dict(full_solve(C.c4(q, nx), f"c4 member {q}, {nx}x{nx}x{nx // 2}"),
                                           member=q)
            print(nx, out["classes"][str(nx)], flush=True)
    else:
        raise SystemExit(f"unknown config {which}")
    with open(os.path.join(HERE, f"{which}_fp64_oracle.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
