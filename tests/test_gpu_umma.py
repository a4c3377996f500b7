"""GPU: the tcgen05 (UMMA) BF16 GEMM of the learned part against numpy.

Inputs are rounded to BF16 on the host; the reference product is formed in
FP64 from the rounded values, so the only difference is the FP32
accumulation order: tolerance 1e-5 relative to sum |a||b|.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_bits(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def bf16_value(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def run(lib, A, a_rs, a_ks, B, b_rs, b_ks, M, N, K, ksplit):
    f = lib.pcf_gemm_bf16
    f.restype = ctypes.c_int
    P16 = ctypes.POINTER(ctypes.c_uint16)
    f.argtypes = [P16, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, P16, ctypes.c_longlong,
                  ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_float)]
    D = np.zeros((M, N), dtype=np.float32)
    rc = f(A.ctypes.data_as(P16), A.size, a_rs, a_ks, B.ctypes.data_as(P16), B.size, b_rs, b_ks, M, N, K, ksplit,
           D.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert rc == 0, rc
    return D


@pytest.mark.parametrize("M,N,K,ksplit,transA,transB", [
    (128, 64, 64, 1, False, False),
    (128, 256, 64, 1, False, False),
    (300, 256, 256, 1, False, False),
    (1000, 64, 256, 1, False, True),
    (256, 256, 4096, 8, True, True),
    (64, 256, 3000, 4, True, True),
    (200, 128, 80, 1, False, False),
])
def test_umma_gemm_matches_numpy(M, N, K, ksplit, transA, transB, pcf):
    lib = pcf.load()
    rng = np.random.default_rng(M * 7 + N + K)
    a = bf16_bits(rng.standard_normal((M, K)))
    b = bf16_bits(rng.standard_normal((N, K)))
    # storage: A(m,k) = A[m*a_rs + k*a_ks]
    if transA:
        As, a_rs, a_ks = np.ascontiguousarray(a.T), 1, M
    else:
        As, a_rs, a_ks = np.ascontiguousarray(a), K, 1
    if transB:
        Bs, b_rs, b_ks = np.ascontiguousarray(b.T), 1, N
    else:
        Bs, b_rs, b_ks = np.ascontiguousarray(b), K, 1
    D = run(lib, As, a_rs, a_ks, Bs, b_rs, b_ks, M, N, K, ksplit)
    ref = bf16_value(a) @ bf16_value(b).T
    scale = np.abs(bf16_value(a)) @ np.abs(bf16_value(b)).T
    assert np.all(np.abs(D - ref) <= 1e-5 * scale + 1e-6), np.max(np.abs(D - ref) / (scale + 1e-30))
