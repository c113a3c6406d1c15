"""Error behaviour of the C ABI on a GPU: rejected arguments return the documented status with a
message (bem_last_error), leave the context's state untouched, and the context stays usable.

The reference reports these cases by exceptions or asserts (std::out_of_range from Triplet and
test_negative, Simulation.hpp asserts); the C ABI returns BEM_ERR_ARG / BEM_ERR_STATE instead.
"""
import ctypes as C

import numpy as np
import pytest

from bem_b200 import _lib as L
from bem_b200 import mesh
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu


def _d(a):
    return a.ctypes.data_as(L._D)


def _i(a):
    return a.ctypes.data_as(L._I64)


@pytest.fixture
def sim():
    v, f = mesh.bubble(3, 1.0, (2.0, 0.0, 0.0))
    s = ColocSim(v, f, solver="lu")
    s.set_phi(0.1 * v[:, 2])
    yield s
    s.close()


def status(sim, rc):
    return rc, sim._L.bem_last_error(sim._h).decode()


def test_rejected_meshes_keep_the_current_one(sim):
    lib, h = sim._L, sim._h
    x0, p0 = sim.get_vertices(), sim.get_phi()
    v, f = mesh.bubble(2, 1.0, (2.0, 0.0, 0.0))
    v = np.ascontiguousarray(v)
    bad = np.array(f, dtype=np.int64)
    bad[3, 1] = len(v)  # index out of range
    assert status(sim, lib.bem_set_mesh(h, len(v), _d(v), len(bad), _i(bad))) == (L.BEM_ERR_ARG,
                                                                                     "triangle index out of range")
    neg = np.array(f, dtype=np.int64)
    neg[0, 0] = -1
    assert lib.bem_set_mesh(h, len(v), _d(v), len(neg), _i(neg)) == L.BEM_ERR_ARG
    lone = np.vstack([v, [[5.0, 0.0, 0.0]]])  # a vertex that belongs to no triangle
    ok = np.array(f, dtype=np.int64)
    rc, msg = status(sim, lib.bem_set_mesh(h, len(lone), _d(lone), len(ok), _i(ok)))
    assert rc == L.BEM_ERR_ARG and "belongs to no triangle" in msg
    assert lib.bem_set_mesh(h, 2, _d(v), len(ok), _i(ok)) == L.BEM_ERR_ARG
    assert lib.bem_set_mesh(h, len(v), _d(v), 0, _i(ok)) == L.BEM_ERR_ARG
    # the mesh and state from before are intact and usable
    assert np.array_equal(sim.get_vertices(), x0) and np.array_equal(sim.get_phi(), p0)
    sim.evolve_system_RK4(1e-3, fixdt=True)
    assert np.all(np.isfinite(sim.get_phi()))


def test_calls_that_need_a_mesh_or_a_batch():
    lib = L.load()
    h = C.c_void_p()
    assert lib.bem_create(C.byref(h), 0, None) == L.BEM_OK
    try:
        G = np.zeros(9)
        assert lib.bem_assemble(h, None, _d(G), None) == L.BEM_ERR_STATE
        assert lib.bem_evolve_rk4(h, 1e-3, 1, None) == L.BEM_ERR_STATE
        assert lib.bem_last_error(h).decode() == "no mesh set"
    finally:
        lib.bem_destroy(h)


def test_argument_checks(sim):
    lib, h, N = sim._L, sim._h, sim.N
    # batch-only calls on a single system
    assert status(sim, lib.bem_evolve_rk4_graph(h, 1e-3, 1))[0] == L.BEM_ERR_STATE
    # pinned count out of range
    assert lib.bem_set_pinned(h, N, 0.2, -0.6, 0.01) == L.BEM_ERR_ARG
    assert lib.bem_set_pinned(h, -1, 0.2, -0.6, 0.01) == L.BEM_ERR_ARG
    # exterior potential with no points
    out = np.zeros(1)
    assert lib.bem_exterior_potential(h, 0, None, None, None, _d(out)) == L.BEM_ERR_ARG
    # null state pointers
    assert lib.bem_set_phi(h, None) == L.BEM_ERR_ARG
    assert lib.bem_position_t(h, None, None, None, None) == L.BEM_ERR_ARG
    # remesh ray casting: no rays is a no-op, bad triangles are rejected
    v = np.ascontiguousarray(sim.get_vertices())
    t = np.zeros((1, 3), dtype=np.int64)
    t[0] = [0, 1, N]
    hit, tri, ok = np.zeros(3), np.zeros(1, dtype=np.int64), np.zeros(1, dtype=np.int32)
    okp = ok.ctypes.data_as(C.POINTER(C.c_int32))
    assert lib.bem_trace_mesh(h, N, _d(v), 1, _i(t), 0, None, None, None, None, None) == L.BEM_OK
    assert lib.bem_trace_mesh(h, N, _d(v), 1, _i(t), 1, _d(hit), _d(hit), _d(hit), _i(tri), okp) == L.BEM_ERR_ARG
    # the context is still usable after every rejection
    sim.evolve_system_RK4(1e-3, fixdt=True)
    assert np.all(np.isfinite(sim.get_vertices()))


def test_trace_mesh_misses_report_triangle_zero(sim):
    # a ray that hits nothing: ok = 0, hit (0, 0, 0), triangle 0, as the reference's caller then sees
    lib, h = sim._L, sim._h
    v = np.ascontiguousarray(sim.get_vertices())
    f = np.ascontiguousarray(mesh.bubble(3, 1.0, (2.0, 0.0, 0.0))[1], dtype=np.int64)
    pos = np.array([[10.0, 10.0, 10.0], [2.0, 0.0, 0.0]])
    d = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    hit, tri, ok = np.full(6, 7.0), np.full(2, 5, dtype=np.int64), np.zeros(2, dtype=np.int32)
    rc = lib.bem_trace_mesh(h, len(v), _d(v), len(f), _i(f), 2, _d(pos), _d(d), _d(hit), _i(tri),
                            ok.ctypes.data_as(C.POINTER(C.c_int32)))
    assert rc == L.BEM_OK
    assert ok[0] == 0 and tri[0] == 0 and np.all(hit[:3] == 0.0)
    # from the centre along z the nearest crossing is at a pole of the sphere (top and bottom are at
    # equal |s| on the symmetric sphere; the first triangle in order is kept)
    assert ok[1] == 1 and abs(abs(hit[5]) - 1.0) < 0.05 and abs(hit[3] - 2.0) < 1e-12 and abs(hit[4]) < 1e-12


def test_expired_barrier_wait_falls_back_to_the_multikernel_bicgstab():
    # A grid-barrier bound of one clock cycle runs out at the persistent BiCGSTAB's first barrier: the
    # kernel sets its error word and returns (no CTA is left waiting), the host counts the expired wait
    # and finishes the solve with the multi-kernel BiCGSTAB, and psi still matches the LU solution.
    # The context keeps the multi-kernel form: a second solve does not try the persistent kernel again.
    v, f = mesh.bubble(6, 1.0, (2.0, 0.0, 0.0))
    phi = 0.1 * np.sin(3 * v[:, 2]) + 0.05 * v[:, 0]
    lu = ColocSim(v, f, solver="lu")
    _, psi_lu = lu.position_t(phi, return_psi=True)
    lu.close()
    s = ColocSim(v, f, solver="bicgstab")
    assert s._L.bem_set_wait_limit(s._h, 0) == L.BEM_ERR_ARG
    assert s._L.bem_set_wait_limit(s._h, 1) == L.BEM_OK
    for k in range(2):
        _, psi = s.position_t(phi, return_psi=True)
        st = s.stats()
        assert st.wait_expired == 1, k
        assert st.last_rel_residual <= 1e-14
        assert np.max(np.abs(psi - psi_lu)) <= 1e-10 * np.max(np.abs(psi_lu))
    s.close()


def test_expired_barrier_wait_in_the_refinement_round_repeats_it_with_separate_launches():
    # With BEM_FLAG_REFINE_PERSISTENT the mixed solve runs each round of refinement steps as one
    # cooperative kernel with grid barriers.  With a one-cycle bound its first barrier wait runs out: the kernel sets its error word
    # and ends, the host counts the expired wait, clears the GEMV tickets and repeats the round with
    # separate GEMV launches (kept for the rest of the context); psi still matches LU.
    v, f = mesh.bubble(8, 1.0, (2.0, 0.0, 0.0))
    phi = 0.1 * np.sin(3 * v[:, 2]) + 0.05 * v[:, 0]
    lu = ColocSim(v, f, solver="lu")
    _, psi_lu = lu.position_t(phi, return_psi=True)
    lu.close()
    s = ColocSim(v, f, solver="mixed")
    s._update(flags=L.FLAG_REFINE_PERSISTENT)
    assert s._L.bem_set_wait_limit(s._h, 1) == L.BEM_OK
    for k in range(2):
        _, psi = s.position_t(phi, return_psi=True)
        assert s.stats().wait_expired == 1, k
        assert np.max(np.abs(psi - psi_lu)) <= 1e-10 * np.max(np.abs(psi_lu))
    s.close()
