import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "pincflow.jl_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def pcf():
    import pincflow_poisson
    pincflow_poisson.load()
    return pincflow_poisson


@pytest.fixture(autouse=True)
def _bounds_checked_build(request):
    """With PCF_LIB_VARIANT=checked (tests/test_gpu_bounds.py runs the GPU
    parity suites that way) every GPU test also requires that the
    bounds-checked library recorded no out-of-range access."""
    yield
    if os.environ.get("PCF_LIB_VARIANT") != "checked" or request.node.get_closest_marker("gpu") is None:
        return
    from pincflow_poisson import _lib
    enabled, site, index = _lib.bounds_check_status()
    assert enabled, "the bounds-checked library is not the one loaded"
    assert site == 0, f"out-of-range access: check site {site}, index {index}"
