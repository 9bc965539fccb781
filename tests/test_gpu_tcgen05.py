"""The split-precision tensor-core product (tcgen05 kind::tf32, 3xTF32
split, FP32 accumulation in tensor memory) through catn_tc_matmul, against
the FP64 product.

Bar: |C - A B| <= 4e-6 * (|A| |B|) elementwise (the 3xTF32 split keeps
about 21 bits of each product and FP32 accumulation adds ~2^-24 per term;
|A| |B| is the product of the absolute values), and a relative Frobenius
error below 2e-6.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def tc_matmul(catn, A, B):
    from catn_b200 import _lib as L
    lib = L.load()
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M, K = A.shape
    N = B.shape[1]
    C = np.zeros((M, N), dtype=np.float64, order="F")
    L.check(lib, lib.catn_tc_matmul(M, N, K, A.ctypes.data_as(ct.c_void_p), B.ctypes.data_as(ct.c_void_p),
                                    C.ctypes.data_as(ct.c_void_p)))
    return C


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (1, 1, 1), (200, 70, 100), (300, 260, 1000), (64, 512, 40),
                                   (1024, 32, 4096)])
def test_tc_matmul_matches_fp64(catn, M, N, K):
    r = np.random.default_rng(M * 7 + N * 3 + K)
    A = r.normal(size=(M, K))
    B = r.normal(size=(K, N))
    C = tc_matmul(catn, A, B)
    ref = A @ B
    bound = np.abs(A) @ np.abs(B)
    assert np.all(np.abs(C - ref) <= 4e-6 * bound + 1e-300)
    assert np.linalg.norm(C - ref) <= 2e-6 * np.linalg.norm(ref)


def test_tc_matmul_graded_columns(catn):
    """Columns spanning twelve decades (the scale of the Jacobi factors the
    split mode feeds it): the error stays relative to each entry's scale."""
    r = np.random.default_rng(5)
    A = r.normal(size=(256, 64)) * np.logspace(0, -12, 64)
    C = tc_matmul(catn, A.T, A)
    ref = A.T @ A
    bound = np.abs(A.T) @ np.abs(A)
    assert np.all(np.abs(C - ref) <= 4e-6 * bound + 1e-300)


def test_tc_matmul_empty_inner_dimension(catn):
    C = tc_matmul(catn, np.zeros((5, 0)), np.zeros((0, 7)))
    assert C.shape == (5, 7) and not C.any()
