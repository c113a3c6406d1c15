"""Pin the oracle (the C restatement, oracle/bem_oracle.c) to the reference's own outputs.

The golden vectors in tests/golden/ref_cases.npz come from the reference sources compiled
here (tests/golden/make_golden.py).  With one thread the reference's arithmetic order is
deterministic and the oracle reproduces it operation for operation, so every comparison
below is bit-exact.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from bem_b200 import mesh

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_cases.npz"))


def _field():
    p_inf, eps, sigma, gamma, amp, omega, phase = GOLD["field"]
    return dict(p_inf=p_inf, epsilon=eps, sigma=sigma, gamma=gamma, amp=amp, omega=omega, phase=phase)


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    assert a.tobytes() == b.tobytes(), f"max |diff| = {np.max(np.abs(a - b))}"


def test_icosphere_matches_reference_generator():
    for nu, digest in zip(GOLD["ico_nus"], GOLD["ico_sha256"]):
        v, f = mesh.icosphere(int(nu))
        h = hashlib.sha256(v.tobytes() + f.astype(np.int64).tobytes()).hexdigest()
        assert h == str(digest), f"nu={nu}"
        assert len(v) == 10 * nu * nu + 2 and len(f) == 20 * nu * nu


@pytest.mark.parametrize("name", ["one", "two"])
@pytest.mark.parametrize("mirror", [0, 1])
def test_assembly_bit_exact(name, mirror):
    v, f = GOLD[f"{name}_verts"], GOLD[f"{name}_trigs"]
    G, H = O.assemble(v, f, bool(mirror))
    same(G, GOLD[f"{name}_G_m{mirror}"])
    same(H, GOLD[f"{name}_H_m{mirror}"])


@pytest.mark.parametrize("name", ["one", "two"])
@pytest.mark.parametrize("mirror", [0, 1])
def test_solve_bit_exact(name, mirror):
    v, f, phi = GOLD[f"{name}_verts"], GOLD[f"{name}_trigs"], GOLD[f"{name}_phi"]
    G, H = O.assemble(v, f, bool(mirror))
    b = O.gemv(H, phi)
    x, _ = O.solve(G, b, use_lu=True)
    same(x, GOLD[f"{name}_psiLU_m{mirror}"])
    x, info = O.solve(G, b, use_lu=False)
    same(x, GOLD[f"{name}_psiBiCG_m{mirror}"])
    assert info["iters"] > 0


def test_four_pi_rule_and_sphere_solution():
    # sum_j H(i,j) = -4 pi for every row (ColocSim.cpp:85-97); constant phi on a sphere
    # gives psi -> -phi/R as the mesh is refined
    v, f = mesh.bubble(4, 1.0, (2.0, 0.0, 0.0))
    G, H = O.assemble(v, f)
    assert np.allclose(H.sum(axis=1), -4 * np.pi, rtol=0, atol=1e-12)
    x, _ = O.solve(G, H @ np.full(len(v), 0.7))
    assert abs(x.mean() + 0.7) < 0.02


def test_position_and_pot_t_bit_exact():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    prm = O.make_params(V0=float(GOLD["two_V0"][0]), **_field())
    vel, _ = O.position_t(v, f, phi, prm)
    same(vel, GOLD["two_vel"])
    same(O.pot_t_multi(v, f, vel, 0.3, prm), GOLD["two_pot_t"])
    prm_s = O.make_params(V0=float(GOLD["two_V0"][0]), **dict(_field(), sigma=0.3))
    same(O.pot_t_multi(v, f, vel, 0.3, prm_s), GOLD["two_pot_t_sigma"])


def _record(S):
    return np.r_[S.x.ravel(), S.phi, S.psi, S.time]


def test_rk4_fixed_lu_bit_exact():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    prm = O.make_params(V0=float(GOLD["two_V0"][0]), **_field())
    S = O.State(v, f, phi)
    for s in range(3):
        S.rk4(1e-2, prm)
        same(_record(S), GOLD["two_rk4"][s])


def test_rk4_adaptive_bicgstab_bit_exact():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    prm = O.make_params(V0=float(GOLD["two_V0"][0]), use_lu=False, **_field())
    S = O.State(v, f, phi)
    for s in range(2):
        S.rk4(0.05, prm, fixdt=False)
        same(_record(S), GOLD["two_rk4_adapt"][s])


def test_euler_bit_exact():
    v, f, phi = GOLD["two_verts"], GOLD["two_trigs"], GOLD["two_phi"]
    prm = O.make_params(V0=float(GOLD["two_V0"][0]), **_field())
    S = O.State(v, f, phi)
    N = len(v)
    for s in range(2):
        S.euler(1e-2, prm)
        same(np.r_[S.x.ravel(), S.phi], GOLD["two_euler"][s][: 4 * N])


def test_wall_image_and_nopenetration_bit_exact():
    v, f = GOLD["wall_verts"], GOLD["wall_trigs"]
    prm = O.make_params(p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, V0=O.volume(v, f), mirror=True)
    S = O.State(v, f, np.full(len(v), 0.6))
    for s in range(2):
        S.rk4(2e-2, prm)
        same(_record(S), GOLD["wall_rk4"][s])


def test_config1_shape_two_steps_bit_exact():
    a = mesh.bubble(7, 1.0, (2.5, 0, 0))
    b = mesh.bubble(7, 1.0, (5.5, 0, 0))
    v, f = mesh.join([a, b])
    n = len(a[0])
    phi = np.r_[np.full(n, -0.5), np.full(n, 0.5)]
    prm = O.make_params(p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, V0=O.volume(v, f))
    S = O.State(v, f, phi)
    for s in range(2):
        S.rk4(1e-3, prm)
        same(_record(S), GOLD["c1_rk4"][s])


def test_negative_x_raises_like_reference():
    v, f = mesh.bubble(1, 1.0, (0.5, 0.0, 0.0))  # crosses the x=0 wall
    S = O.State(v, f, np.zeros(len(v)))
    with pytest.raises(IndexError):
        S.rk4(1e-3, O.make_params(V0=1.0))


def test_exterior_potential_bit_exact():
    # compute_exterior_pot (LinLinSim.cpp:440-477) with a given psi, and exterior_pot (assemble,
    # LU solve, compute_exterior_pot) restated with the oracle's own assembly and LU
    v, f = GOLD["two_verts"], GOLD["two_trigs"]
    phi = GOLD["two_phi"]
    pts, psi = GOLD["ext_points"], GOLD["ext_psi"]
    assert np.array_equal(O.exterior_pot(v, f, phi, psi, pts), GOLD["ext_direct"])
    G, H = O.assemble(v, f)
    psi_l, _ = O.solve(G, O.gemv(H, phi), use_lu=True)
    assert np.array_equal(O.exterior_pot(v, f, phi, psi_l, pts), GOLD["ext_solve"])


def test_config1_first_25_of_100_steps_bit_exact():
    # the oracle against the reference's own 100-step trajectory of the same set-up
    # (tests/golden/c1_100.npz), up to its first stored record, step 25, bit for bit
    c1 = np.load(os.path.join(os.path.dirname(__file__), "golden", "c1_100.npz"))
    assert int(c1["steps"][0]) == 25
    a = mesh.bubble(7, 1.0, (2.5, 0, 0))
    b = mesh.bubble(7, 1.0, (5.5, 0, 0))
    v, f = mesh.join([a, b])
    n = len(a[0])
    prm = O.make_params(p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, V0=O.volume(v, f))
    S = O.State(v, f, np.r_[np.full(n, -0.5), np.full(n, 0.5)])
    for s in range(25):
        S.rk4(1e-3, prm)
    same(_record(S), c1["records"][0])
