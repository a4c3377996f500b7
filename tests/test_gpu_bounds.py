"""GPU: the parity suites on the bounds-checked build.

The library built with -DPCF_BOUNDS_CHECK (build.py --checked) checks the
global indices of its stencil, Thomas, multigrid transfer, assembly and
corrector kernels against their arrays' extents; an access out of range is
skipped and recorded, never a fault.  This test runs the operator, solver,
multigrid, corrector and predictor parity suites (small grids: 40x1x40 up to
512x10x8, odd sizes, partial tiles) in a child process that loads that
library (PCF_LIB_VARIANT=checked); there every test also asserts that no
access was out of range (tests/conftest.py), on top of its elementwise
comparison with the oracle.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SUITES = ["test_gpu_parity.py", "test_gpu_multigrid.py", "test_gpu_corrector.py", "test_gpu_predictor.py",
          "test_gpu_lhs.py"]


def test_parity_suites_on_the_bounds_checked_build():
    lib = os.path.join(os.path.dirname(HERE), "pincflow.jl_b200", "lib", "libpincflow_poisson_checked.so")
    assert os.path.exists(lib), "build the checked library first (pincflow.jl_b200/build.py --checked)"
    env = dict(os.environ, PCF_LIB_VARIANT="checked")
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"] + \
          [os.path.join(HERE, s) for s in SUITES]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1200, cwd=os.path.dirname(HERE))
    print(r.stdout[-3000:], r.stderr[-2000:])
    assert r.returncode == 0, r.stdout[-3000:]
