"""The batched complex GEMM through the C ABI: the FP64 tensor path against
NumPy (1e-13 relative) and the 3xTF32 tcgen05 path against NumPy (error below
1e-5 of |A||B| summed over K: the 3xTF32 error with FP32 accumulation over K up to 882)."""
import numpy as np
import pytest

import openrcwa_b200 as o

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("M,N,K,b", [(1, 1, 1, 1), (17, 5, 9, 2), (128, 128, 32, 2), (130, 257, 200, 3),
                                     (300, 64, 882, 2)])
def test_gemm_fp64_and_tf32x3(eng, M, N, K, b):
    rng = np.random.default_rng(M + N + K)
    A, B, C = crand(rng, b, M, K), crand(rng, b, K, N), crand(rng, b, M, N)
    alpha, beta = 0.7 - 0.2j, -1.3 + 0.4j
    ref = alpha * (A @ B) + beta * C
    scale = (np.abs(A) @ np.abs(B)) * abs(alpha)
    D64 = eng.zgemm(A, B, C, alpha, beta, o.RCWA_PREC_FP64)
    assert np.max(np.abs(D64 - ref) / (scale + np.abs(beta * C))) < 1e-13
    Dtc = eng.zgemm(A, B, C, alpha, beta, o.RCWA_PREC_MIXED)
    assert np.max(np.abs(Dtc - ref) / (scale + np.abs(beta * C))) < 1e-5


def test_gemm_tf32x3_without_c(eng):
    rng = np.random.default_rng(9)
    A, B = crand(rng, 4, 150, 70), crand(rng, 4, 70, 140)
    D = eng.zgemm(A, B, precision=o.RCWA_PREC_MIXED)
    assert np.max(np.abs(D - A @ B) / (np.abs(A) @ np.abs(B))) < 1e-5


def test_gemm_tf32x3_outside_fp32_range(eng):
    # operands far outside the FP32 range are scaled by powers of two first
    rng = np.random.default_rng(11)
    A, B = crand(rng, 2, 96, 80) * 1e50, crand(rng, 2, 80, 70) * 1e-60
    D = eng.zgemm(A, B, precision=o.RCWA_PREC_MIXED)
    assert np.all(np.isfinite(D))
    assert np.max(np.abs(D - A @ B) / (np.abs(A) @ np.abs(B))) < 1e-5
