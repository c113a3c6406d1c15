"""The pinned-contact-line variant (the reference's ColocSimPin) on the GPU.

* Assembly: with pinned vertices the matrices are the plain collocation matrices (wall image on) with
  the pinned columns exchanged, G(:,j) = -H(:,j) and H(:,j) = -G(:,j) (ColocSimPin.cpp:113-117), bit for
  bit.
* position_t: the solve and the pinned vertices' drift velocity and potential against numpy on the
  same matrices (the stored psi stands in for the potential at the pinned vertices; vertex normals as
  generate_vertex_normals, Mesh.cpp:141-159); tolerance 1e-10 relative.
* Trajectory: RK4 (fixed and adaptive dt) and Euler steps of a hemisphere on the wall against the
  reference's own ColocSimPin built on the CPU (tests/golden/pinned_check, oracle/pinned_check.cpp's first
  block): positions, phi and psi to the float32 precision of the export, time, volume and the pinned
  vertices' positions and potential to 1e-9; the mixed-precision solver to 1e-8 of the FP64 LU path.
"""
import os

import numpy as np
import pytest

from bem_b200 import mesh
from bem_b200.sim import ColocSim, ColocSimPin, _on_wall, move_flagged_to_end
from plyio import read_ply

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "pinned_check")
PHYS = dict(p_inf=1.0, epsilon=1.4, sigma=0.0, gamma=1.4)
FIELD = (-0.3, 0.7, 0.0, 0.2)  # -0.3 sin(0.2 x + 0.7 t), the driver's field


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def vertex_normals(x, f):
    acc = np.zeros_like(x)
    for t in f:
        for k in range(3):
            a, b, c = t[k], t[(k + 1) % 3], t[(k + 2) % 3]
            B, C = x[b] - x[a], x[c] - x[a]
            acc[a] += np.cross(B, C) * (1.0 / (B.dot(B) * C.dot(C)))
    return acc / np.linalg.norm(acc, axis=1)[:, None]


def wall_cap32(nu):
    # the wall cap as the reference's drivers read it from a PLY file: float32 coordinates
    v, f = mesh.wall_cap(nu)
    return v.astype(np.float32).astype(np.float64), f


def permuted_trigs(nu):
    # the constructor's renumbering of the wall cap's triangles
    v, f = wall_cap32(nu)
    return move_flagged_to_end(v, f, _on_wall)[1]


def pinned_sim(nu=6, solver="lu", **kw):
    v, f = wall_cap32(nu)
    return ColocSimPin(v, f, pressurefield=FIELD, solver=solver, **PHYS, **kw)


def test_assembly_exchanges_pinned_columns():
    sp = pinned_sim(5)
    n = sp.N_pin
    assert n == 20
    x = sp.get_vertices()
    assert np.all(x[-n:, 0] == 0.0) and np.all(x[:-n, 0] > 1e-3)
    plain = ColocSim(x, permuted_trigs(5), mirror=True, **PHYS)
    G0, H0 = plain.assemble_matrices()
    G, H = sp.assemble_matrices()
    assert np.array_equal(G[:, :-n], G0[:, :-n]) and np.array_equal(H[:, :-n], H0[:, :-n])
    assert np.array_equal(G[:, -n:], -H0[:, -n:]) and np.array_equal(H[:, -n:], -G0[:, -n:])


def test_position_t_solves_exchanged_system_and_drifts():
    sp = pinned_sim(5)
    n, N = sp.N_pin, sp.N
    rng = np.random.default_rng(4)
    psi = 0.1 * rng.standard_normal(N)
    sp.set_psi(psi)
    x = sp.get_vertices()
    pot = 0.05 + 0.02 * rng.standard_normal(N)
    pot_in = pot.copy()
    G, H = sp.assemble_matrices()
    vel, psil = sp.position_t(pot, return_psi=True)
    # right-hand side with the stored psi at the pinned vertices
    q = pot_in.copy()
    q[-n:] = psi[-n:]
    sol = np.linalg.solve(G, H @ q)
    assert rel(psil, sol) <= 1e-10
    assert np.array_equal(pot[:-n], pot_in[:-n])
    assert np.array_equal(pot[-n:], psil[-n:])  # solved potential written back (PotVec&)
    nv = vertex_normals(x, permuted_trigs(5))
    beta, ceq, cnl = sp.drift
    for i in range(N - n, N):
        c = nv[i, 0]
        w = np.array([0.0, nv[i, 1], nv[i, 2]])
        w /= np.linalg.norm(w)
        d = beta * (ceq - c) + cnl * (c * c * c) / (c * c - 1.0)
        assert np.allclose(vel[i], w * d, rtol=0, atol=1e-12)
        assert vel[i, 0] == 0.0


def golden_lines(block):
    blk, pins = None, []
    for ln in open(os.path.join(GOLD, "ref_stdout.txt")):
        w = ln.split()
        if w[0] == "block" and int(w[1]) == block:
            blk = dict(time=float(w[3]), volume=float(w[5]), verts=int(w[7]), npin=int(w[9]))
        elif w[0] == "pinned" and int(w[1]) == block:
            pins.append([float(u) for u in w[3:]])
    return blk, np.array(pins)


def first_block(solver):
    sp = pinned_sim(6, solver=solver)
    sp.set_phi(np.full(sp.N, 0.05))
    sp.set_min_dt(5e-3)
    sp.evolve_system_RK4(2e-3, fixdt=True)
    sp.evolve_system_RK4(2e-3, fixdt=False)
    sp.evolve_system(2e-3, fixdt=False)
    return sp


def test_trajectory_matches_reference_colocsimpin():
    sp = first_block("lu")
    blk, pins = golden_lines(0)
    assert sp.N == blk["verts"] and sp.N_pin == blk["npin"]
    assert abs(sp.get_time() - blk["time"]) <= 1e-9 * blk["time"]
    assert abs(sp.get_volume() - blk["volume"]) <= 1e-9 * blk["volume"]
    x, phi = sp.get_vertices(), sp.get_phi()
    n = sp.N_pin
    assert rel(x[-n:], pins[:, :3]) <= 1e-9
    assert rel(phi[-n:], pins[:, 3]) <= 1e-9
    xr, er, tr = read_ply(os.path.join(GOLD, "ref-0.ply"))
    assert np.array_equal(permuted_trigs(6), tr)
    assert np.max(np.abs(x - xr)) <= 1e-6
    assert np.max(np.abs(phi - er["phi"])) <= 1e-6 * np.max(np.abs(er["phi"]))
    assert np.max(np.abs(sp.get_psi() - er["psi"])) <= 1e-6 * np.max(np.abs(er["psi"]))


def test_mixed_solver_matches_lu_with_pins():
    a, b = first_block("lu"), first_block("mixed")
    assert rel(b.get_vertices(), a.get_vertices()) <= 1e-8
    assert rel(b.get_phi(), a.get_phi()) <= 1e-8
    assert rel(b.get_psi(), a.get_psi()) <= 1e-8


def test_pins_refused_where_unsupported():
    sp = pinned_sim(3, solver="mixed")
    with pytest.raises(Exception):
        sp._check(sp._L.bem_adjoint_record(sp._h, 1e-3, 1))
    with pytest.raises(Exception):
        sp._check(sp._L.bem_set_pinned(sp._h, sp.N, *sp.drift))
    # batches of independent bubbles take no pins
    from bem_b200.batch import BubbleBatch
    bb = BubbleBatch([mesh.bubble(3, 1.0, (2.0, 0.0, 0.0)), mesh.bubble(2, 0.5, (1.5, 0.0, 0.0))])
    assert bb._L.bem_set_pinned(bb._h, 2, *sp.drift) != 0


def test_new_mesh_clears_the_pins():
    # bem_set_mesh starts without pinned vertices (the pinned count refers to a vertex order)
    import ctypes as C
    from bem_b200 import _lib as L
    sp = pinned_sim(3)
    v, f = wall_cap32(3)
    vv, ff = np.ascontiguousarray(v), np.ascontiguousarray(f, dtype=np.int64)
    sp._check(sp._L.bem_set_mesh(sp._h, len(vv), vv.ctypes.data_as(L._D), len(ff), ff.ctypes.data_as(L._I64)))
    n = C.c_int64(-1)
    sp._check(sp._L.bem_get_pinned(sp._h, C.byref(n)))
    assert n.value == 0
