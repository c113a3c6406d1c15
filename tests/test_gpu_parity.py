"""Parity of the CUDA path (through the C ABI) with the reference.

Small cases compare against the golden vectors produced by the reference's own code
(tests/golden/ref_cases.npz) and against the oracle (the bit-exact C restatement) on the same
seeded inputs; full-size cases check size-independent properties (the 4 pi row-sum rule, the
analytic sphere solution, agreement of the three solvers).

Tolerance: relative error max|gpu - ref| / max|ref| <= 1e-10, the FP64 path's parity bar.  The
GPU contracts multiply-adds into FMAs and uses the hardware reciprocal square root, so the
agreement is at the 1e-15 level per entry rather than bit-exact.
"""
import os

import numpy as np
import pytest

import oracle as O
from bem_b200 import mesh
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_cases.npz"))
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _field():
    p_inf, eps, sigma, gamma, amp, omega, phase = GOLD["field"]
    return dict(p_inf=p_inf, epsilon=eps, sigma=sigma, gamma=gamma), (amp, omega, phase)


@pytest.mark.parametrize("name", ["one", "two"])
@pytest.mark.parametrize("mirror", [0, 1])
def test_assembly_matches_reference(name, mirror):
    v, f = GOLD[f"{name}_verts"], GOLD[f"{name}_trigs"]
    sim = ColocSim(v, f, mirror=bool(mirror))
    G, H = sim.assemble_matrices()
    assert rel(G, GOLD[f"{name}_G_m{mirror}"]) < 1e-13
    assert rel(H, GOLD[f"{name}_H_m{mirror}"]) < 1e-13


def test_assembly_nu10_matches_oracle_and_is_reproducible():
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f)
    G, H = sim.assemble_matrices()
    G2, H2 = sim.assemble_matrices()
    assert G.tobytes() == G2.tobytes() and H.tobytes() == H2.tobytes()  # no atomics: bit-reproducible
    Go, Ho = O.assemble(v, f)
    assert rel(G, Go) < 1e-13 and rel(H, Ho) < 1e-13


def _uv_sphere(nlon, nlat, center):
    # closed UV sphere, outward orientation; the two poles have valence nlon
    v = [[0.0, 0.0, 1.0]]
    for a in range(1, nlat):
        th = np.pi * a / nlat
        for o in range(nlon):
            ph = 2 * np.pi * o / nlon
            v.append([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    v.append([0.0, 0.0, -1.0])
    f = []
    ring = lambda a, o: 1 + (a - 1) * nlon + o % nlon
    for o in range(nlon):
        f.append([0, ring(1, o), ring(1, o + 1)])
        for a in range(1, nlat - 1):
            f.append([ring(a, o), ring(a + 1, o), ring(a + 1, o + 1)])
            f.append([ring(a, o), ring(a + 1, o + 1), ring(a, o + 1)])
        f.append([ring(nlat - 1, o), len(v) - 1, ring(nlat - 1, o + 1)])
    return np.array(v) + np.array(center), np.array(f, dtype=np.int64)


@pytest.mark.parametrize("mirror", [0, 1])
def test_assembly_high_valence_vertex_matches_oracle(mirror):
    # poles of valence 40: the singular pass takes the triangles around a vertex 32 at a time, so a
    # ring of 40 spans two chunks; G, H and the right-hand side against the oracle
    v, f = _uv_sphere(40, 9, (2.0, 0.0, 0.0))
    assert mesh.signed_volume(v, f) > 0
    sim = ColocSim(v, f, mirror=bool(mirror))
    G, H = sim.assemble_matrices()
    Go, Ho = O.assemble(v, f, mirror=bool(mirror))
    assert rel(G, Go) < 1e-13 and rel(H, Ho) < 1e-13
    # the fused right-hand side: psi from the device solve against the oracle's matrices
    phi = 0.1 * np.sin(2 * v[:, 2]) + 0.05 * v[:, 1]
    _, psi = sim.position_t(phi, return_psi=True)
    assert rel(psi, np.linalg.solve(Go, Ho @ phi)) < 1e-10


@pytest.mark.parametrize("cg", ["16", "32", "48", "64"])
def test_assembly_tile_shapes_agree(cg, monkeypatch):
    # every column-group width of the tile kernel gives the same matrices (two bubbles, nu=7)
    monkeypatch.setenv("BEM_ASM_CG", cg)
    a = mesh.bubble(7, 1.0, (2.5, 0, 0))
    b = mesh.bubble(7, 0.8, (4.9, 0, 0))
    v, f = mesh.join([a, b])
    G, H = ColocSim(v, f, mirror=True).assemble_matrices()
    Go, Ho = O.assemble(v, f, True)
    assert rel(G, Go) < 1e-13 and rel(H, Ho) < 1e-13


def test_assembly_full_size_four_pi_rule():
    # N = 4002 (icosphere nu=20): sum_j H(i,j) = -4 pi for every row (ColocSim.cpp:85-97)
    v, f = mesh.bubble(20, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f)
    G, H = sim.assemble_matrices()
    assert np.max(np.abs(H.sum(axis=1) + 4 * np.pi)) < 1e-10
    assert np.all(np.isfinite(G)) and np.all(np.diag(G) > 0)


@pytest.mark.parametrize("solver", ["lu", "bicgstab", "mixed"])
def test_solvers_match_reference(solver):
    for name in ("one", "two"):
        v, f, phi = GOLD[f"{name}_verts"], GOLD[f"{name}_trigs"], GOLD[f"{name}_phi"]
        sim = ColocSim(v, f, solver=solver)
        G, H = sim.assemble_matrices()
        x = sim.solve_system(G, H @ phi)
        assert rel(x, GOLD[f"{name}_psiLU_m0"]) < TOL, solver


def test_sphere_known_answer_full_size():
    # constant phi on a sphere of radius R: dphi/dn -> -phi/R (exterior Dirichlet problem)
    v, f = mesh.bubble(20, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f, solver="lu")
    vel, psi = sim.position_t(np.full(len(v), 0.7), return_psi=True)
    assert abs(psi.mean() + 0.7) < 2e-3
    sim.set_solver("mixed")
    _, psi_m = sim.position_t(np.full(len(v), 0.7), return_psi=True)
    sim.set_solver("bicgstab")
    _, psi_b = sim.position_t(np.full(len(v), 0.7), return_psi=True)
    assert rel(psi_m, psi) < 1e-9 and rel(psi_b, psi) < 1e-9


def test_position_and_pot_t_match_reference():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, fld = _field()
    sim = ColocSim(v, f, pressurefield=fld, solver="lu", **phys)
    sim.set_V_0(float(GOLD["two_V0"][0]))
    vel = sim.position_t(phi)
    assert rel(vel, GOLD["two_vel"]) < TOL
    assert rel(sim.pot_t_multi(vel, 0.3), GOLD["two_pot_t"]) < TOL
    sim_s = ColocSim(v, f, pressurefield=fld, solver="lu", **dict(phys, sigma=0.3))
    sim_s.set_V_0(float(GOLD["two_V0"][0]))
    assert rel(sim_s.pot_t_multi(vel, 0.3), GOLD["two_pot_t_sigma"]) < TOL


def _record(sim):
    return np.r_[sim.get_vertices().ravel(), sim.get_phi(), sim.get_psi(), sim.get_time()]


def test_rk4_fixed_dt_matches_reference():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, fld = _field()
    sim = ColocSim(v, f, pressurefield=fld, solver="lu", **phys)
    sim.set_V_0(float(GOLD["two_V0"][0]))
    sim.set_phi(phi)
    for s in range(3):
        sim.evolve_system_RK4(1e-2, fixdt=True)
        assert rel(_record(sim), GOLD["two_rk4"][s]) < TOL


def test_rk4_adaptive_bicgstab_matches_reference():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, fld = _field()
    sim = ColocSim(v, f, pressurefield=fld, solver="bicgstab", **phys)
    sim.set_V_0(float(GOLD["two_V0"][0]))
    sim.set_phi(phi)
    for s in range(2):
        sim.evolve_system_RK4(0.05, fixdt=False)
        assert rel(_record(sim), GOLD["two_rk4_adapt"][s]) < TOL


def test_rk4_mixed_solver_matches_reference():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, fld = _field()
    sim = ColocSim(v, f, pressurefield=fld, solver="mixed", **phys)
    sim.set_V_0(float(GOLD["two_V0"][0]))
    sim.set_phi(phi)
    for s in range(3):
        sim.evolve_system_RK4(1e-2, fixdt=True)
        assert rel(_record(sim), GOLD["two_rk4"][s]) < 1e-9


def test_euler_matches_reference():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, fld = _field()
    sim = ColocSim(v, f, pressurefield=fld, solver="lu", **phys)
    sim.set_V_0(float(GOLD["two_V0"][0]))
    sim.set_phi(phi)
    N = len(v)
    for s in range(2):
        sim.evolve_system(1e-2, fixdt=True)
        got = np.r_[sim.get_vertices().ravel(), sim.get_phi()]
        assert rel(got, GOLD["two_euler"][s][: 4 * N]) < TOL


def test_wall_image_and_nopenetration_match_reference():
    v, f = GOLD["wall_verts"], GOLD["wall_trigs"]
    sim = ColocSim(v, f, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, solver="lu", mirror=True)
    sim.set_phi(np.full(len(v), 0.6))
    for s in range(2):
        sim.evolve_system_RK4(2e-2, fixdt=True)
        assert rel(_record(sim), GOLD["wall_rk4"][s]) < TOL


def test_config1_shape_matches_reference():
    a = mesh.bubble(7, 1.0, (2.5, 0, 0))
    b = mesh.bubble(7, 1.0, (5.5, 0, 0))
    v, f = mesh.join([a, b])
    n = len(a[0])
    phi = np.r_[np.full(n, -0.5), np.full(n, 0.5)]
    sim = ColocSim(v, f, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, solver="lu")
    sim.set_phi(phi)
    for s in range(2):
        sim.evolve_system_RK4(1e-3, fixdt=True)
        assert rel(_record(sim), GOLD["c1_rk4"][s]) < TOL


def test_field_callback_equals_device_field():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    phys, (amp, omega, phase) = _field()
    dev = ColocSim(v, f, pressurefield=(amp, omega, phase), solver="lu", **phys)
    host = ColocSim(v, f, pressurefield=lambda x, t: amp * np.sin(omega * t + phase), solver="lu", **phys)
    for s in (dev, host):
        s.set_phi(phi)
        s.set_time(0.4)
        s.evolve_system_RK4(1e-2, fixdt=True)
    assert rel(_record(dev), _record(host)) < 1e-13


def test_negative_x_raises_like_reference():
    v, f = mesh.bubble(2, 1.0, (0.5, 0.0, 0.0))
    sim = ColocSim(v, f)
    with pytest.raises(IndexError):
        sim.evolve_system_RK4(1e-3, fixdt=True)


@pytest.mark.parametrize("nu", [4, 9, 16])
def test_persistent_bicgstab_matches_multikernel_and_lu(nu):
    # the cooperative-kernel BiCGSTAB and its multi-kernel form run the same iteration; both reach
    # the machine-precision residual and agree with the FP64 LU solution
    from bem_b200 import _lib as L
    v, f = mesh.bubble(nu, 1.0, (2.0, 0.0, 0.0))
    rng = np.random.default_rng(nu)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None]
    phi = 0.1 * np.sin(3 * v[:, 2]) + 0.05 * v[:, 0]
    _, psi_lu = ColocSim(v, f, solver="lu").position_t(phi, return_psi=True)
    one = ColocSim(v, f, solver="bicgstab")
    many = ColocSim(v, f, solver="bicgstab")
    many._update(flags=L.FLAG_BICGSTAB_MULTIKERNEL)
    for sim in (one, many):
        _, psi = sim.position_t(phi, return_psi=True)
        st = sim.stats()
        assert rel(psi, psi_lu) <= TOL
        assert st.last_rel_residual <= 1e-14 and 0 < st.last_iters <= 2 * len(v)


def test_mixed_solver_falls_back_on_singular_system():
    # G with two equal columns (rank N - 1) and a consistent right-hand side: no approximate inverse
    # exists, and the mixed solve hands over to the FP64 BiCGSTAB (the reference's solver) instead of
    # failing
    v, f = mesh.bubble(4, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f, solver="mixed")
    G, _ = sim.assemble_matrices()
    G[:, 1] = G[:, 0]
    b = G @ np.random.default_rng(2).standard_normal(len(v))
    x = sim.solve_system(G, b)
    assert sim.stats().fp64_fallbacks >= 1
    assert np.linalg.norm(G @ x - b) <= 1e-8 * np.linalg.norm(b)


def test_mixed_solver_steps_bubble_cut_by_its_wall_image():
    # a bubble centred on the wall plane with the wall image on (the reference's oscillations driver
    # as shipped): G = S + S R nearly annihilates the modes odd in x.  Euler steps (no x < 0 check, as
    # in the reference) go through, on the mixed path or its FP64 fallback.
    v, f = mesh.bubble(4, 1.0, (0.0, 0.0, 0.0))
    sim = ColocSim(v, f, mirror=True, solver="mixed")
    sim.set_phi(0.05 + 0.01 * v[:, 2])
    for _ in range(3):
        sim.evolve_system(1e-3, fixdt=True)
    assert np.all(np.isfinite(sim.get_vertices())) and np.all(np.isfinite(sim.get_phi()))


def test_state_in_one_call_each_way():
    v, f = mesh.bubble(4, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f)
    rng = np.random.default_rng(1)
    x = v + 0.01 * rng.standard_normal(v.shape)
    phi, psi = rng.standard_normal(len(v)), rng.standard_normal(len(v))
    sim.set_state(x, phi, psi, time=0.25)
    gx, gp, gs, gt = sim.get_state()
    assert np.array_equal(gx, x) and np.array_equal(gp, phi) and np.array_equal(gs, psi) and gt == 0.25
    sim.set_state(phi=2 * phi)  # the other parts stay
    gx, gp, gs, gt = sim.get_state()
    assert np.array_equal(gx, x) and np.array_equal(gp, 2 * phi) and np.array_equal(gs, psi) and gt == 0.25
    assert np.array_equal(sim.get_vertices(), x) and np.array_equal(sim.get_phi(), 2 * phi)


def test_negative_x_leaves_the_state_untouched():
    # the reference's test_negative throws before the step changes anything (LinLinSim.cpp:198)
    v, f = mesh.bubble(3, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f, solver="mixed")
    x = v.copy()
    x[5, 0] = -0.01
    phi = 0.1 * v[:, 1]
    sim.set_state(x, phi, np.zeros(len(v)), time=1.0)
    with pytest.raises(IndexError):
        sim.evolve_system_RK4(1e-3, fixdt=True)
    gx, gp, gs, gt = sim.get_state()
    assert np.array_equal(gx, x) and np.array_equal(gp, phi) and np.all(gs == 0.0) and gt == 1.0


@pytest.mark.parametrize("mirror", [False, True])
def test_stage_predictor_keeps_the_trajectory(mirror):
    # the mixed solver starts each RK4 stage from an extrapolation of the same stage of earlier steps,
    # with the first residual b - G x0 formed by the assembly; any start converges to the same FP64
    # solution, so the trajectory equals the one started from the previous stage with the residual
    # from a GEMV (BEM_FLAG_NO_STAGE_PREDICTOR), also after the state is pushed back unchanged (history
    # kept) or changed (history dropped), and with an adaptive step
    from bem_b200 import _lib as L
    v, f = mesh.bubble(8, 1.0, (2.0, 0.0, 0.0))
    rng = np.random.default_rng(3)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None]
    sims = [ColocSim(v, f, pressurefield=(-0.8, 2 * np.pi / 5, 0.0), solver="mixed", mirror=mirror)
            for _ in range(2)]
    sims[1]._update(flags=L.FLAG_NO_STAGE_PREDICTOR)
    for sim in sims:
        sim.set_phi(0.0)
        for _ in range(6):
            sim.evolve_rk4_steps(5e-3, 1)
        x, p, s = sim.get_vertices(), sim.get_phi(), sim.get_psi()
        sim.set_state(x, p, s)  # the same state: the predictor's history stays
        sim.evolve_system_RK4(5e-3, fixdt=True)
        x, p, s = sim.get_vertices(), sim.get_phi(), sim.get_psi()
        sim.set_state(x, 1.001 * p, s)  # another state: the history is dropped
        for _ in range(4):
            sim.evolve_system_RK4(5e-3, fixdt=False)
    (xa, pa), (xb, pb) = [(sim.get_vertices(), sim.get_phi()) for sim in sims]
    assert rel(xa, xb) < 1e-11 and rel(pa, pb) < 1e-11
    assert sims[0].stats().total_iters > 0 and sims[0].stats().solves == sims[1].stats().solves


def test_solution_consumers_enqueued_again_after_a_second_round():
    # the velocity and Dphi/Dt of a stage are enqueued behind the solve's first round; when the
    # tolerance tightens mid-run (and the predictor's history is dropped), the first round no longer
    # suffices and they are enqueued again with the final solution: the trajectory still follows the
    # FP64 LU path
    v, f = mesh.bubble(6, 1.0, (2.0, 0.0, 0.0))
    fld = (-0.8, 2 * np.pi / 5, 0.0)
    mix = ColocSim(v, f, pressurefield=fld, solver="mixed")
    ref = ColocSim(v, f, pressurefield=fld, solver="lu")
    for sim in (mix, ref):
        sim.set_phi(0.1 * v[:, 2])
    for k in range(8):
        if k == 4:
            mix._update(mixed_tol=1e-13)
        for sim in (mix, ref):
            sim.evolve_system_RK4(5e-3, fixdt=True)
    assert rel(mix.get_vertices(), ref.get_vertices()) < 1e-10
    assert rel(mix.get_phi(), ref.get_phi()) < 1e-10


def test_mixed_precision_error_headline_size():
    # N = 4002 (config 2 mesh with the seeded 1% radial perturbation): psi of the mixed path
    # against the FP64 LU path at <= 1e-8 relative
    v, f = mesh.bubble(20, 1.0, (0.0, 0.0, 0.0))
    rng = np.random.default_rng(0)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None] + np.array([2.0, 0.0, 0.0])
    phi = 0.1 * np.sin(3 * v[:, 2])
    ref = ColocSim(v, f, solver="lu")
    _, psi_ref = ref.position_t(phi, return_psi=True)
    mix = ColocSim(v, f, solver="mixed")
    _, psi_mix = mix.position_t(phi, return_psi=True)
    assert rel(psi_mix, psi_ref) <= 1e-8


def test_exterior_potential_matches_reference():
    # compute_exterior_pot with a given psi, and exterior_pot (LU solve first) against the reference
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    sim = ColocSim(v, f, solver="lu")
    sim.set_phi(phi)
    pts, psi = GOLD["ext_points"], GOLD["ext_psi"]
    assert rel(sim.exterior_potential(pts, phi=phi, psi=psi), GOLD["ext_direct"]) <= 1e-12
    assert rel(sim.exterior_potential(pts), GOLD["ext_solve"]) <= TOL


def test_exterior_potential_grid_matches_oracle():
    # nu = 10 bubble, 300 seeded points on shells around it (outside and inside)
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    rng = np.random.default_rng(11)
    phi = 0.1 * np.sin(2 * v[:, 1]) + 0.02 * v[:, 0]
    psi = 0.05 * np.cos(v[:, 2])
    d = rng.standard_normal((300, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    r = np.where(np.arange(300) % 3 == 0, 0.5, rng.uniform(1.2, 4.0, 300))
    pts = np.array([2.0, 0.0, 0.0]) + d * r[:, None]
    sim = ColocSim(v, f)
    got = sim.exterior_potential(pts, phi=phi, psi=psi)
    assert rel(got, O.exterior_pot(v, f, phi, psi, pts)) <= 1e-12


def test_refinement_round_kernel_equals_separate_launches():
    # the mixed solve's refinement round as one cooperative kernel and as separate GEMV launches: the
    # same tiles, per-thread order and split sums, so whole RK4 trajectories agree bit for bit (the
    # separate launches without the gated extra steps, which the round kernel does not issue)
    from bem_b200 import _lib as L
    v, f = mesh.bubble(12, 1.0, (2.0, 0.0, 0.0))
    rng = np.random.default_rng(3)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None]
    out = []
    for flags in (L.FLAG_NO_IR_GATE, L.FLAG_REFINE_PERSISTENT):
        sim = ColocSim(v, f, pressurefield=(-0.8, 2 * np.pi / 5, 0.0), solver="mixed", p_inf=1.0, epsilon=1.0,
                       gamma=1.4)
        sim._update(flags=flags)
        sim.set_phi(0.0)
        for _ in range(4):
            sim.evolve_system_RK4(5e-3, fixdt=True)
        x, p, s, t = sim.get_state()
        out.append((x.tobytes(), p.tobytes(), s.tobytes(), t, sim.stats().total_iters))
        sim.close()
    assert out[0] == out[1]


def test_mixed_solve_gated_extra_steps_end_in_one_round():
    # the first round of each refinement appends gated steps (a device check applies the host's
    # convergence rule and the GEMVs after it return at once): along a smooth trajectory nearly every
    # solve ends in one round, every solve meets the refinement tolerance, and the trajectory equals
    # the FP64 BiCGSTAB one
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    phys = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)
    mix = ColocSim(v, f, solver="mixed", pressurefield=(-0.8, 2.0 * np.pi / 5.0, 0.0), **phys)
    ref = ColocSim(v, f, solver="bicgstab", pressurefield=(-0.8, 2.0 * np.pi / 5.0, 0.0), **phys)
    for sim in (mix, ref):
        sim.set_phi(0.05 * np.cos(v[:, 2]))
    s0 = mix.stats()
    for _ in range(10):
        mix.evolve_system_RK4(5e-3, fixdt=True)
        ref.evolve_system_RK4(5e-3, fixdt=True)
        assert mix.stats().last_rel_residual <= 1e-12
    s1 = mix.stats()
    solves = s1.solves - s0.solves
    assert solves == 40
    assert s1.ir_rounds - s0.ir_rounds <= solves + 4
    assert rel(mix.get_psi(), ref.get_psi()) <= 1e-8
    assert rel(mix.get_vertices(), ref.get_vertices()) <= 1e-10
