"""GPU: the allocation-free dot product (pcf_global_dot_noalloc) agrees with
the handle-based entry point (pcf_global_dot).

The allocation-free variant serves callers that cannot let the library
allocate device memory (a host model whose GPU memory is held by its own
pool allocator, or a step recorded into a CUDA graph); it keeps its scratch
in a fixed __device__ array.  The test calls it twice in a row through the C
ABI, so it also checks that the second call starts from clean scratch.  This
file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.pcf_global_dot_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p]
    return f


@pytest.mark.parametrize("shape", [(40, 48, 64), (96, 128, 256)])
def test_noalloc_dot_matches_handle_dot_twice(shape, pcf):
    import torch

    from pincflow_poisson.fields import Domain

    noalloc = _bind(pcf.load())
    nz, ny, nx = shape
    n = nx * ny * nz
    rng = np.random.default_rng(77)
    with pcf.PoissonSolver(Domain(nx, ny, nz)) as s:
        for call in range(2):
            a = rng.standard_normal(shape)
            b = rng.standard_normal(shape) * (1 + call)
            ref = s.compute_global_dot_product(a, b)
            da = torch.from_numpy(a).cuda()
            db = torch.from_numpy(b).cuda()
            out = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = noalloc(da.data_ptr(), db.data_ptr(), n, out.data_ptr(), None)
            assert rc == 0, pcf._lib.strerror(rc)
            torch.cuda.synchronize()
            got = float(out.item())
            assert abs(got - ref) <= 1e-12 * np.abs(a * b).sum(), (call, got, ref)


def test_noalloc_rejects_bad_sizes(pcf):
    noalloc = _bind(pcf.load())
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert noalloc(None, None, 5, out.data_ptr(), None) == pcf._lib.PCF_EINVAL
    assert noalloc(None, None, -1, out.data_ptr(), None) == pcf._lib.PCF_EINVAL
    big = 268_435_456 + 1
    assert noalloc(out.data_ptr(), out.data_ptr(), big, out.data_ptr(), None) == pcf._lib.PCF_ERANGE
    # n = 0: the empty sum
    out.fill_(3.0)
    assert noalloc(None, None, 0, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert float(out.item()) == 0.0
