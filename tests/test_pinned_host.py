"""Host side of the pinned-contact-line variant, no GPU: the vertex renumbering of the reference's
ColocSimPin::set_x_boundary (ColocSimPin.cpp:257-287), restated in bem_b200.sim.move_flagged_to_end,
against the reference's own build (tests/golden/pinned_check/ref-0.ply carries the reference's numbering:
its first block only steps, so the triangles are the constructor's), and the wall cap mesh."""
import os
from collections import Counter

import numpy as np

from bem_b200 import mesh
from bem_b200.sim import _on_wall, move_flagged_to_end
from plyio import read_ply

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pinned_check")


def test_wall_cap_contact_line_on_the_wall():
    for nu in (1, 3, 6):
        v, f = mesh.wall_cap(nu, radius=1.5)
        assert len(v) == 2 * nu * nu + 2 * nu + 1 and len(f) == 4 * nu * nu
        assert np.allclose(np.linalg.norm(v, axis=1), 1.5, rtol=0, atol=1e-15)
        edges = Counter(tuple(sorted((t[k], t[(k + 1) % 3]))) for t in f for k in range(3))
        assert set(edges.values()) <= {1, 2}
        boundary = [e for e, c in edges.items() if c == 1]
        assert len(boundary) == 4 * nu and all(v[a, 0] == 0.0 and v[b, 0] == 0.0 for a, b in boundary)
        assert mesh.signed_volume(v, f) > 0.0  # outward orientation


def test_set_x_boundary_numbering_matches_reference():
    v, f = mesh.wall_cap(6)
    phi = np.arange(len(v), dtype=np.float64)
    v2, t2, origin, n, phi2 = move_flagged_to_end(v, f, _on_wall, phi)
    assert n == 24
    assert np.all(v2[-n:, 0] == 0.0) and np.all(np.abs(v2[:-n, 0]) >= 1e-5)
    assert np.array_equal(phi2, phi[origin]) and np.array_equal(v2, v[origin])
    _, _, tr = read_ply(os.path.join(GOLD, "ref-0.ply"))
    assert np.array_equal(t2, tr)


def test_flagged_scan_reexamines_swapped_in_vertex():
    # flags (carried in z) at 0, 1 and the last two: the vertex that trades places with vertex k-1 is
    # examined again before the scan moves on (the reference's i--, k-- step)
    v = np.zeros((6, 3))
    v[:, 1] = np.arange(6)
    v[:, 2] = [1, 1, 0, 0, 1, 1]
    f = np.array([[0, 1, 2], [3, 4, 5]])
    v2, t2, origin, n = move_flagged_to_end(v, f, lambda vv, i: vv[i, 2] == 1.0)
    assert n == 4
    assert list(origin) == [3, 2, 1, 4, 5, 0]
    assert np.array_equal(v2[:, 1], origin) and np.array_equal(v2[:, 2], [0, 0, 1, 1, 1, 1])
    assert t2.tolist() == [[5, 2, 1], [0, 3, 4]]
