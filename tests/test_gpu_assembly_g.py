"""The G-only assembly of the step path (triangle patches, no H matrix) against the oracle.

position_t (LinLinSim.cpp:26-83) needs G and b = H*phi after the 4 pi rule (ColocSim.cpp:85-97), never
H itself.  The step path forms them with the triangle-patch kernels: every regular pair is evaluated
once, columns shared between patches are summed from halo columns, and b comes out as
sum_j H(i, j) (phi_j - phi_i) - 4 pi phi_i.  bem_assemble_rhs returns what the step path formed.

Tolerances: G entry-wise 1e-13 relative to max|G| (the FP64 assembly bar); b 1e-12 relative to
max|b| (the oracle forms H*phi from the assembled H, a different summation of the same terms);
states of trajectories through both kernels 1e-12.
"""
import numpy as np
import pytest

import bench
import oracle as O
from bem_b200 import _lib as L
from bem_b200 import mesh
from bem_b200.sim import ColocSim

from test_gpu_parity import _uv_sphere

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def check_against_oracle(v, f, phi, mirror=False):
    sim = ColocSim(v, f, mirror=mirror)
    G, b = sim.assemble_rhs(phi)
    G2, b2 = sim.assemble_rhs(phi)
    sim.close()
    assert G.tobytes() == G2.tobytes() and b.tobytes() == b2.tobytes()  # no atomics: bit-reproducible
    Go, Ho = O.assemble(v, f, mirror=mirror)
    assert rel(G, Go) <= 1e-13
    assert rel(b, Ho @ phi) <= 1e-12


@pytest.mark.parametrize("mirror", [False, True])
def test_g_only_assembly_two_bubbles(mirror):
    a = mesh.bubble(7, 1.0, (2.5, 0, 0))
    b = mesh.bubble(7, 0.8, (4.9, 0, 0))
    v, f = mesh.join([a, b])
    phi = 0.1 * np.sin(2 * v[:, 1]) + 0.03 * v[:, 0]
    check_against_oracle(v, f, phi, mirror)


@pytest.mark.parametrize("mirror", [False, True])
def test_g_only_assembly_high_valence(mirror):
    # poles of valence 40: a patch holding a pole's ring would touch 41 vertices, so the planner
    # splits it below the 32 columns a patch may hold
    v, f = _uv_sphere(40, 9, (2.0, 0.0, 0.0))
    phi = 0.1 * np.sin(2 * v[:, 2]) + 0.05 * v[:, 1]
    check_against_oracle(v, f, phi, mirror)


@pytest.mark.parametrize("nu", [1, 2])
def test_g_only_assembly_smallest_meshes(nu):
    v, f = mesh.bubble(nu, 1.0, (2.0, 0.0, 0.0))
    check_against_oracle(v, f, 0.2 + 0.1 * v[:, 2])


def test_g_only_assembly_headline_size():
    v, f = bench.workload()
    phi = 0.1 * np.sin(3 * v[:, 2])
    check_against_oracle(v, f, phi)


def test_step_path_with_and_without_h_agree():
    # the same RK4 trajectory with the G-only kernel and with the bem_assemble kernel on the step path
    a = mesh.bubble(6, 1.0, (2.5, 0, 0))
    b = mesh.bubble(5, 0.7, (4.6, 0, 0))
    v, f = mesh.join([a, b])
    phi = np.r_[np.full(len(a[0]), -0.4), np.full(len(b[0]), 0.2)]
    sims = []
    for flags in (0, L.FLAG_STEP_ASSEMBLE_H):
        s = ColocSim(v, f, pressurefield=bench.FIELD, solver="lu", **bench.PHYS)
        s._update(flags=flags)
        s.set_phi(phi)
        for _ in range(3):
            s.evolve_system_RK4(1e-2, fixdt=True)
        sims.append(s.get_state())
        s.close()
    (x0, p0, s0, t0), (x1, p1, s1, t1) = sims
    assert t0 == t1
    assert rel(x0, x1) <= 1e-12 and rel(p0, p1) <= 1e-12 and rel(s0, s1) <= 1e-12
