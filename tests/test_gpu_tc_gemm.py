"""The split-precision tensor-core GEMM (tcgen05, bf16 hi/lo operands, FP32 accumulation) that
refreshes the mixed solver's approximate inverse, checked against an FP64 product.

BF16x3 keeps about 16 significant bits per operand (hi + lo) and drops the lo*lo term, so the
relative error of each product entry is bounded by a few times 2^-16 of the magnitude of the terms;
tolerance here: max |C - C64| <= 4e-5 * max_ij (|A| |B|)_ij.
"""
import ctypes as C

import numpy as np
import pytest

from bem_b200 import _lib as L

pytestmark = pytest.mark.gpu


def run(A, B):
    n = A.shape[0]
    A32 = np.asfortranarray(A, dtype=np.float32)
    B32 = np.asfortranarray(B, dtype=np.float32)
    out = np.empty((n, n), dtype=np.float32, order="F")
    fp = C.POINTER(C.c_float)
    rc = L.load().bem_gemm_bf16x3(0, n, A32.ctypes.data_as(fp), B32.ctypes.data_as(fp), out.ctypes.data_as(fp))
    assert rc == L.BEM_OK
    return out, A32.astype(np.float64) @ B32.astype(np.float64), np.abs(A32.astype(np.float64)) @ np.abs(B32.astype(np.float64))


@pytest.mark.parametrize("n", [256, 300, 1000, 4002])
def test_bf16x3_gemm_matches_fp64(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, n))
    Cg, C64, Cabs = run(A, B)
    assert np.max(np.abs(Cg - C64)) <= 4e-5 * np.max(Cabs)


def test_bf16x3_gemm_identity_and_layout():
    n = 384
    rng = np.random.default_rng(1)
    B = rng.standard_normal((n, n))
    Cg, C64, _ = run(np.eye(n), B)
    # I * B: only the split of B matters -> ~2^-16 relative per entry, and the layout is exact
    assert np.max(np.abs(Cg - C64) / (np.abs(C64) + 1e-30)) < 2e-5
    A = rng.standard_normal((n, n))
    Cg, C64, _ = run(A, np.eye(n))
    assert np.max(np.abs(Cg - C64) / (np.abs(C64) + 1e-30)) < 2e-5
