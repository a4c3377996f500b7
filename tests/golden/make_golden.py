"""Generates tests/golden/small_cases.npz from the CPU oracle.

The reference (Julia) cannot run here and ships no known-answer data for its
Poisson path, so these fixtures pin the oracle itself: any later change of
the oracle or of the input generators that moves these numbers fails
tests/test_oracle_kat.py, and the GPU tests compare against them without
running the oracle.  Inputs are regenerated from seeds by
pincflow_poisson.configs; only outputs are stored.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "pincflow.jl_b200"), os.path.dirname(HERE)]

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402

from golden_cases import GOLDEN, golden_case  # noqa: E402


def main():
    out = {}
    for name in GOLDEN:
        cfg = golden_case(name)
        dom, f = cfg["dom"], cfg["fields"]
        d = O.dims(dom.nx, dom.ny, dom.nz, dom.nbx)
        coef = O.compute_operator(d, O.MODELS[cfg["model"]], f, cfg["rho"], cfg["betar"], cfg["dt"],
                                  cfg["rayleigh_factor"], cfg["damp"], cfg["p"])
        x = np.random.default_rng(21).standard_normal(dom.interior_shape)
        out[f"{name}/coef"] = coef
        out[f"{name}/apply_total"] = O.apply_operator(d, coef, x, False)
        out[f"{name}/apply_horizontal"] = O.apply_operator(d, coef, x, True)
        out[f"{name}/precond"] = O.apply_preconditioner(d, coef, f["dx"], f["dy"], 1.0, 2, x)
        b = O.apply_operator(d, coef, np.random.default_rng(22).standard_normal(dom.interior_shape))
        sol, info = O.bicgstab(d, coef, f["dx"], f["dy"], b, tolerance=1e-12, tolerance_is_relative=True,
                               poisson_iterations=1000)
        out[f"{name}/rhs"] = b
        out[f"{name}/solution"] = sol
        out[f"{name}/niter"] = np.array(info["niter"])
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
