"""The FP64 LU solve (the reference's PartialPivLU option, Simulation.cpp:57-60) on general matrices.

The collocation G of a smooth bubble rarely needs a row interchange, so these tests hand the solver
seeded Gaussian matrices, which pivot at almost every column, and compare with numpy's LAPACK solve.
Sizes cover one panel, a partial last panel, several panels and the headline size (N = 4002, the
cluster panel with 16 CTAs and the tensor-core trailing update); the unit lower and upper triangular
solves run over blocks of 64 rows.
"""
import numpy as np
import pytest

from bem_b200 import mesh
from bem_b200.sim import ColocSim
import bem_b200._lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative error of the solution; Gaussian matrices have cond ~ N, so kappa*eps ~ 1e-12


def _sim(nu):
    v, f = mesh.bubble(nu, 1.0, (2.0, 0.0, 0.0))
    return ColocSim(v, f, solver="lu")


@pytest.mark.parametrize("nu", [1, 2, 4, 7, 16, 20])
def test_lu_solves_pivoting_matrices_like_lapack(nu):
    sim = _sim(nu)
    n = sim.N
    rng = np.random.default_rng(100 + nu)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    b = rng.standard_normal(n)
    x = sim.solve_system(A, b)
    ref = np.linalg.solve(A, b)
    err = np.max(np.abs(x - ref)) / np.max(np.abs(ref))
    assert err <= TOL, (n, err)
    # the residual of a backward-stable factorisation
    res = np.linalg.norm(A @ x - b) / (np.linalg.norm(A, 1) * np.linalg.norm(x))
    assert res <= 1e-14, (n, res)


def test_lu_repeated_solves_are_bit_identical():
    sim = _sim(16)
    n = sim.N
    rng = np.random.default_rng(7)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    b = rng.standard_normal(n)
    x1 = sim.solve_system(A, b)
    x2 = sim.solve_system(A, b)
    assert np.array_equal(x1, x2)


def test_lu_ties_and_row_interchanges_of_a_permutation_matrix():
    # a permuted diagonal: every pivot is the unique nonzero of its column, found by the interchanges
    sim = _sim(4)
    n = sim.N
    rng = np.random.default_rng(3)
    p = rng.permutation(n)
    A = np.zeros((n, n), order="F")
    A[p, np.arange(n)] = 1.0 + np.arange(n) / n
    b = rng.standard_normal(n)
    x = sim.solve_system(A, b)
    assert np.allclose(x, np.linalg.solve(A, b), rtol=0, atol=1e-14)


def test_lu_reports_a_zero_pivot():
    sim = _sim(2)
    n = sim.N
    A = np.ones((n, n), order="F")  # rank one
    with pytest.raises(L.BemError) as e:
        sim.solve_system(A, np.ones(n))
    assert e.value.code == L.BEM_ERR_SINGULAR
    # the context stays usable
    rng = np.random.default_rng(5)
    B = np.asfortranarray(rng.standard_normal((n, n)))
    c = rng.standard_normal(n)
    assert np.allclose(sim.solve_system(B, c), np.linalg.solve(B, c), rtol=1e-10, atol=0)


def test_lu_cluster_panel_wait_expiry_falls_back():
    # the cluster panel's mbarrier waits are bounded by the context's wait limit; at one clock cycle
    # they run out, the kernel records the error word and still makes every write and arrival, the
    # host counts it and factors again with the single-CTA panel, and the solution is still right
    sim = _sim(20)
    n = sim.N
    rng = np.random.default_rng(11)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    b = rng.standard_normal(n)
    assert sim._L.bem_set_wait_limit(sim._h, 1) == L.BEM_OK
    x = sim.solve_system(A, b)
    assert sim.stats().wait_expired >= 1
    ref = np.linalg.solve(A, b)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= TOL
    # later solves of the context keep the single-CTA panel
    x2 = sim.solve_system(A, b)
    assert np.array_equal(x, x2)


def test_lu_panels_taller_than_a_cluster_use_the_grid_barrier_panel():
    # N = 6762 (icosphere nu = 26): the first panels hold more rows than one thread-block cluster's
    # shared memory, so they run on co-resident CTAs with grid barriers (their interchanges composed by
    # a separate kernel), and the later, shorter panels on the cluster
    sim = _sim(26)
    n = sim.N
    assert n == 6762
    rng = np.random.default_rng(17)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    b = rng.standard_normal(n)
    x = sim.solve_system(A, b)
    ref = np.linalg.solve(A, b)
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= TOL
    assert sim.stats().wait_expired == 0
