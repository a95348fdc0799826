"""tcgen05 building blocks: one tensor-core GEMM tile against numpy.

D[128][N] = A[128][K] B[N][K]^T with A and B rounded to BF16 and FP32
accumulation in tensor memory; the reference is the same product of the
BF16-rounded operands in FP64 (tolerance: FP32 accumulation, 1e-5 of the
largest |D|)."""
import ctypes

import numpy as np
import pytest

from ct2_b200 import _lib
from oracle import learned as OL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(32, 16), (32, 96), (64, 64), (64, 32)])
def test_tc_gemm_tile(gpu, N, K):
    rng = np.random.Generator(np.random.PCG64(N * 100 + K))
    A = rng.normal(0, 1, (128, K)).astype(np.float32)
    B = rng.normal(0, 1, (N, K)).astype(np.float32)
    D = np.zeros((128, N), np.float32)
    lib = _lib.load()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.ct2g_tc_selftest(0, p(A), p(B), N, K, p(D))
    assert rc == 0, _lib.load().ct2g_status_string(rc)
    ref = OL.bf16_round(A).astype(np.float64) @ OL.bf16_round(B).astype(np.float64).T
    assert np.abs(D - ref).max() <= 1e-5 * np.abs(ref).max()
