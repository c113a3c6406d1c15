"""Batches of independent bubbles (block-diagonal systems) against the single-bubble path.

Every bubble of a batch must follow exactly what a single-bubble simulation of it does: the
batched assembly computes each block with the same per-pair arithmetic and the same column groups,
so its G and H blocks equal the single-bubble matrices bit for bit; RK4 trajectories agree to the
solver tolerance (both sides refine to a 1e-12 relative residual, so states agree to ~1e-10); a step
replayed from the captured CUDA graph equals the same step issued kernel by kernel, bit for bit.
"""
import numpy as np
import pytest

from bem_b200 import mesh
from bem_b200.batch import BubbleBatch
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def sweep(nus, seed=0):
    """Bubbles of a radius x pressure sweep: icosphere nu, radius R0 at (R0 + 1, 0, 0), 1% radial
    perturbation, amplitude and period per bubble."""
    rng = np.random.default_rng(seed)
    meshes, prm = [], []
    for nu in nus:
        R0 = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        v, f = mesh.bubble(nu, 1.0, (0.0, 0.0, 0.0))
        v = v * (R0 * (1.0 + 0.01 * rng.standard_normal(len(v))))[:, None] + np.array([R0 + 1.0, 0.0, 0.0])
        A, T = rng.uniform(0.1, 1.5), rng.uniform(2.0, 10.0)
        meshes.append((v, f))
        prm.append((-A, 2 * np.pi / T))
    return meshes, prm


PHYS = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)


def make_batch(meshes, prm):
    bb = BubbleBatch(meshes, **PHYS)
    bb.set_block_params(amp=[p[0] for p in prm], omega=[p[1] for p in prm])
    return bb


def test_batched_blocks_equal_single_assembly():
    meshes, prm = sweep([2, 4, 3, 5, 2])
    bb = make_batch(meshes, prm)
    blocks = bb.assemble_blocks()
    for (v, f), (Gb, Hb) in zip(meshes, blocks):
        G, H = ColocSim(v, f, **PHYS).assemble_matrices()
        assert np.array_equal(Gb, G)
        assert np.array_equal(Hb, H)


def test_block_params_default_to_own_volume():
    meshes, prm = sweep([3, 4, 2])
    bb = make_batch(meshes, prm)
    p = bb.block_params()
    for b, (v, f) in enumerate(meshes):
        assert p["V0"][b] == pytest.approx(mesh.signed_volume(v, f), rel=1e-12)
        assert p["amp"][b] == prm[b][0] and p["omega"][b] == prm[b][1]


@pytest.mark.parametrize("graph", [False, True])
def test_batched_rk4_matches_single_bubbles(graph):
    meshes, prm = sweep([4, 3, 6, 2, 5, 4])
    dt, steps = 2e-3, 3
    bb = make_batch(meshes, prm)
    # nonzero potential so that the first solve is not trivial
    phi = np.concatenate([0.05 * np.sin(2 * v[:, 2]) for v, _ in meshes])
    bb.set_phi(phi)
    if graph:
        bb.evolve_graph(dt, steps)
    else:
        bb.evolve_rk4_steps(dt, steps)
    X, P, S = bb.get_vertices(), bb.get_phi(), bb.get_psi()
    for b, ((v, f), (amp, om)) in enumerate(zip(meshes, prm)):
        sim = ColocSim(v, f, pressurefield=(amp, om, 0.0), solver="lu", **PHYS)
        sim.set_phi(phi[bb.block(b)])
        for _ in range(steps):
            sim.evolve_system_RK4(dt, fixdt=True)
        sl = bb.block(b)
        assert rel(X[sl], sim.get_vertices()) <= 1e-10
        assert rel(P[sl], sim.get_phi()) <= 1e-9
        assert rel(S[sl], sim.get_psi()) <= 1e-9
    assert abs(bb.get_time() - steps * dt) < 1e-15
    rho, res, _ = bb.block_stats()
    assert np.all(res <= 1e-12)


def test_graph_replay_equals_plain_steps():
    meshes, prm = sweep([3, 5, 4, 2])
    a, b = make_batch(meshes, prm), make_batch(meshes, prm)
    phi = np.concatenate([0.03 * np.cos(3 * v[:, 0]) for v, _ in meshes])
    a.set_phi(phi)
    b.set_phi(phi)
    a.evolve_rk4_steps(2e-3, 4)
    b.evolve_graph(2e-3, 2)
    b.evolve_graph(2e-3, 2)
    assert np.array_equal(a.get_vertices(), b.get_vertices())
    assert np.array_equal(a.get_phi(), b.get_phi())
    assert np.array_equal(a.get_psi(), b.get_psi())


def test_autotune_keeps_state_and_results():
    meshes, prm = sweep([6, 4, 5, 3, 7])
    a, b = make_batch(meshes, prm), make_batch(meshes, prm)
    phi = np.concatenate([0.02 * v[:, 1] for v, _ in meshes])
    a.set_phi(phi)
    b.set_phi(phi)
    a.evolve_graph(2e-3, 1)
    b.evolve_graph(2e-3, 1)
    x0, p0, t0 = b.get_vertices(), b.get_phi(), b.get_time()
    V0 = b.block_params()["V0"]
    cg, ms = b.autotune()
    assert cg in (16, 32, 48, 64) and np.all(ms > 0)
    assert np.array_equal(b.get_vertices(), x0) and np.array_equal(b.get_phi(), p0) and b.get_time() == t0
    assert np.array_equal(b.block_params()["V0"], V0)
    a.evolve_graph(2e-3, 2)
    b.evolve_graph(2e-3, 2)
    # another tile shape sums the triangles of a column in another order: agreement to rounding
    assert rel(b.get_vertices(), a.get_vertices()) <= 1e-12
    assert rel(b.get_phi(), a.get_phi()) <= 1e-10


def test_zero_potential_first_step():
    # phi = 0 gives a zero right-hand side in the first stage (x = 0 without refinement)
    meshes, prm = sweep([3, 2, 4])
    bb = make_batch(meshes, prm)
    bb.evolve_graph(2e-3, 2)
    for b, ((v, f), (amp, om)) in enumerate(zip(meshes, prm)):
        sim = ColocSim(v, f, pressurefield=(amp, om, 0.0), solver="lu", **PHYS)
        sim.evolve_rk4_steps(2e-3, 2)
        assert rel(bb.get_phi()[bb.block(b)], sim.get_phi()) <= 1e-9
