"""The mixed solver's approximate inverse built by blocked Gauss-Jordan elimination with row partial
pivoting in FP32, its rank-64 updates as split-precision tcgen05 GEMMs, then polished by
Newton-Schulz steps.  Whatever the approximate inverse, the mixed solve refines against the FP64
matrix, so its answers are checked against FP64 solutions: 1e-9 relative for a random matrix
(cond ~ 1e3), 1e-10 for the BEM system (the parity bar).
"""
import numpy as np
import pytest

import bench
from bem_b200 import _lib as L
from bem_b200 import mesh
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_gj_inverse_solves_a_matrix_that_needs_pivoting():
    # a Gaussian random matrix: partial pivoting interchanges rows at almost every column, and
    # N = 1002 ends with a panel of 42 columns
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    n = len(v)
    rng = np.random.default_rng(5)
    G = np.asfortranarray(rng.standard_normal((n, n)))
    b = rng.standard_normal(n)
    sim = ColocSim(v, f, solver="mixed")
    sim._update(flags=L.FLAG_INVERSE_GJ)
    x = sim.solve_system(G, b)
    st = sim.stats()
    sim.close()
    assert st.gj_inverses == 1 and st.fp64_fallbacks == 0 and st.gmres_fallbacks == 0
    assert rel(x, np.linalg.solve(G, b)) <= 1e-9


def test_gj_and_newton_schulz_inverses_give_the_same_solution():
    # the headline mesh (N = 4002): psi of the mixed solve through either set-up of the inverse
    v, f = bench.workload()
    phi = 0.1 * np.sin(3 * v[:, 2])
    out = {}
    for name, flags in (("gj", L.FLAG_INVERSE_GJ), ("ns", L.FLAG_INVERSE_NS)):
        sim = ColocSim(v, f, solver="mixed")
        sim._update(flags=flags)
        _, psi = sim.position_t(phi, return_psi=True)
        out[name] = (psi, sim.stats())
        sim.close()
    assert out["gj"][1].gj_inverses == 1 and out["ns"][1].gj_inverses == 0
    assert out["gj"][1].fp64_fallbacks == 0 and out["gj"][1].gmres_fallbacks == 0
    assert rel(out["gj"][0], out["ns"][0]) <= 1e-10
