"""The allocation-free GEMM entry point (bem_gemm_bf16x3_noalloc) against the allocating one.

Callers that cannot allocate GPU memory themselves (a framework owning the device heap, loops that
must not allocate after start-up, plug-ins handed only device pointers) use the no-alloc form: it
takes device pointers for A, B and C and keeps its scratch in a static device array.  This file is
collected last on purpose (test_zz_*): a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from bem_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_N = 1024  # BEM_NOALLOC_GEMM_MAX_N in include/bem_b200.h


def allocating(A, B):
    n = A.shape[0]
    fp = C.POINTER(C.c_float)
    out = np.empty((n, n), dtype=np.float32, order="F")
    rc = L.load().bem_gemm_bf16x3(0, n, A.ctypes.data_as(fp), B.ctypes.data_as(fp), out.ctypes.data_as(fp))
    assert rc == L.BEM_OK
    return out


def no_alloc(A, B):
    import torch

    n = A.shape[0]
    # the test owns the device buffers; the entry point itself allocates nothing
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major A: store A^T row-major
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dC = torch.empty((n, n), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.load().bem_gemm_bf16x3_noalloc(0, n, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                          C.c_void_p(dC.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == L.BEM_OK
    torch.cuda.synchronize()
    return dC.cpu().numpy().T  # back to the (row, column) view of the column-major result


@pytest.mark.parametrize("n", [300, MAX_N])
def test_no_alloc_gemm_matches_allocating_gemm_twice(n):
    rng = np.random.default_rng(7 + n)
    for call in range(2):  # two calls in a row share the same scratch
        A = np.asfortranarray(rng.standard_normal((n, n)), dtype=np.float32)
        B = np.asfortranarray(rng.standard_normal((n, n)), dtype=np.float32)
        ref = allocating(A, B)
        got = no_alloc(A, B)
        scale = np.max(np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64)))
        # the tolerance of the GEMM tests (tests/test_gpu_tc_gemm.py)
        assert np.max(np.abs(got - ref)) <= 4e-5 * scale, call
        exact = A.astype(np.float64) @ B.astype(np.float64)
        assert np.max(np.abs(got - exact)) <= 4e-5 * scale, call


def test_no_alloc_rejects_sizes_beyond_the_scratch():
    lib = L.load()
    rc = lib.bem_gemm_bf16x3_noalloc(0, MAX_N + 1, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == L.BEM_ERR_ARG
