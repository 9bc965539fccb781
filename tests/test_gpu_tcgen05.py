"""The split-precision tensor-core product (tcgen05 kind::tf32, 3xTF32
split, FP32 accumulation in tensor memory) through catn_tc_matmul, against
the FP64 product.

Bar: |C - A B| <= 4e-6 * (|A| |B|) elementwise, where |A| |B| is the
product of the absolute values, and the Frobenius norm of the error below
1e-6 of that of |A| |B|.  The 3xTF32 split represents each operand to about
2^-22 (the lo part is itself rounded to TF32), so each product carries
~2^-21 relative error; FP32 accumulation adds ~2^-24 per term.  Errors are
relative to |A| |B|, not to A B, whose entries cancel.
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
    assert np.linalg.norm(C - ref) <= 1e-6 * np.linalg.norm(bound)


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
