"""Why the mixed-precision path assembles G and H in FP64 (CPU, oracle only).

The error bar of the mixed path is 1e-8 relative in dphi/dn against the FP64 solution.  Rounding the
exact FP64 matrices to FP32 once -- the best an FP32 assembly could do -- already moves the solution
by more than that on the bubble meshes of the benchmarks (cond(G) ~ 1e2), so the assembly stays FP64
and the FP32 precision goes into the approximate inverse of the solve only, where refinement
against the FP64 G removes its error."""
import numpy as np

import oracle as O
from bem_b200 import mesh


def test_fp32_rounded_matrices_miss_the_error_bar():
    v, f = mesh.bubble(10, 1.0, (0.0, 0.0, 0.0))
    rng = np.random.default_rng(0)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None] + np.array([2.0, 0.0, 0.0])
    G, H = O.assemble(v, f)
    phi = 0.1 * np.sin(3 * v[:, 2]) + 0.05
    psi = np.linalg.solve(G, H @ phi)
    r32 = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
    psi32 = np.linalg.solve(r32(G), r32(H) @ phi)
    err = np.max(np.abs(psi32 - psi)) / np.max(np.abs(psi))
    assert err > 1e-8  # measured 3.4e-7 at N = 1002 (cond(G) = 94)
    # iterative refinement against the FP64 G with an FP32 inverse recovers the FP64 solution
    X = r32(np.linalg.inv(G))
    x = np.zeros_like(psi)
    b = H @ phi
    for _ in range(6):
        x = x + X @ (b - G @ x)
    assert np.max(np.abs(x - psi)) / np.max(np.abs(psi)) <= 1e-12
