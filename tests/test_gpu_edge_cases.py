"""Edge cases of the CUDA path against the oracle (the C restatement of the reference): the smallest
closed meshes (a tetrahedron, N = 4; the icosphere nu = 1, N = 12), a mesh whose vertex order is
shuffled (ragged column groups), and the three solvers on them.  Below one column group of the
assembly tiles and below one row tile, every kernel runs its boundary paths.  Tolerance 1e-10
relative (1e-9 for the mixed solver, whose answer is the FP64 solution to a 1e-12 residual)."""
import numpy as np
import pytest

import oracle as O
from bem_b200 import mesh
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def tetrahedron():
    v = np.array([[1.0, 1.0, 1.0], [1.0, -1.0, -1.0], [-1.0, 1.0, -1.0], [-1.0, -1.0, 1.0]]) * 0.5
    f = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]])
    return v + np.array([2.0, 0.0, 0.0]), f


def shuffled(nu, seed=3):
    v, f = mesh.bubble(nu, 1.0, (2.0, 0.0, 0.0))
    perm = np.random.default_rng(seed).permutation(len(v))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(v))
    return v[perm], inv[f]


CASES = {"tetrahedron": tetrahedron, "ico1": lambda: mesh.bubble(1, 1.0, (2.0, 0.0, 0.0)),
         "shuffled_ico5": lambda: shuffled(5)}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("mirror", [False, True])
def test_small_meshes_assembly_matches_oracle(case, mirror):
    v, f = CASES[case]()
    G, H = ColocSim(v, f, mirror=mirror).assemble_matrices()
    Go, Ho = O.assemble(v, f, mirror=mirror)
    assert rel(G, Go) <= TOL and rel(H, Ho) <= TOL
    # the 4 pi rule: every row of H sums to -4 pi (with the image, the image's solid angle enters)
    if not mirror:
        assert np.allclose(H.sum(axis=1), -4 * np.pi, rtol=0, atol=1e-9)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("solver", ["lu", "bicgstab", "mixed"])
def test_small_meshes_rk4_matches_oracle(case, solver):
    v, f = CASES[case]()
    phi = 0.2 + 0.05 * v[:, 2]
    prm = O.make_params(p_inf=1.0, epsilon=1.2, gamma=1.4, V0=O.volume(v, f), amp=-0.3, omega=1.1,
                        use_lu=True)
    st = O.State(v, f, phi)
    sim = ColocSim(v, f, p_inf=1.0, epsilon=1.2, gamma=1.4, pressurefield=(-0.3, 1.1, 0.0), solver=solver)
    sim.set_phi(phi)
    tol = 1e-9 if solver == "mixed" else TOL
    for _ in range(3):
        st.rk4(2e-3, prm)
        sim.evolve_system_RK4(2e-3, fixdt=True)
        assert rel(sim.get_vertices(), st.x) <= tol
        assert rel(sim.get_phi(), st.phi) <= tol
        assert rel(sim.get_psi(), st.psi) <= tol
