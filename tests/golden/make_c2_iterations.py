"""Runs the CPU oracle's FP64 BiCGSTAB (the reference algorithm) on the full
256 x 256 x 128 pseudo-incompressible workload to relative residual 1e-10 and
records the iteration count, the final residual and the run time in
tests/golden/c2_fp64_oracle.json.  Takes several minutes on 8 cores.

Usage: python tests/golden/make_c2_iterations.py
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


def main():
    cfg = C.c2()
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
    out = dict(workload="c2 256x256x128 PseudoIncompressible seed 12345", niter=info["niter"],
               errflag=info["errflag"], residual=float(info["residual"]), true_residual=true_res,
               seconds_assembly=t1 - t0, seconds_bicgstab=t2 - t1, threads=O.get_threads(),
               solution_rms=float(np.sqrt((sol ** 2).mean())),
               solution_checksum=float(np.abs(sol).sum()))
    with open(os.path.join(HERE, "c2_fp64_oracle.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
