"""Asynchronous PLY export: the files hold exactly what Simulation::export_mesh would write for the
state at the call (export_ply_float layout, MeshIO.cpp:263-298), although the simulation keeps
stepping while they are copied and written."""
import numpy as np
import pytest

from bem_b200 import mesh
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu


def reference_layout(x, tri, phi, psi):
    """Bytes of export_ply_float for this state."""
    head = ("ply\nformat binary_little_endian 1.0\ncomment Output from BEM simulation\n"
            f"element vertex {len(x)}\nproperty float x\nproperty float y\nproperty float z\n"
            "property float phi\nproperty float psi\n"
            f"element face {len(tri)}\nproperty list uchar uint vertex_indices\nend_header\n").encode()
    v = np.zeros(len(x), dtype=[("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("phi", "<f4"), ("psi", "<f4")])
    v["x"], v["y"], v["z"], v["phi"], v["psi"] = x[:, 0], x[:, 1], x[:, 2], phi, psi
    fc = np.zeros(len(tri), dtype=[("n", "u1"), ("i", "<u4", (3,))])
    fc["n"] = 3
    fc["i"] = tri
    return head + v.tobytes() + fc.tobytes()


def test_async_export_matches_state_at_call(tmp_path):
    v, f = mesh.bubble(6, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f, epsilon=1.0, gamma=1.4, pressurefield=(-0.5, 1.0, 0.0), solver="mixed")
    sim.set_phi(0.02 * np.sin(3 * v[:, 2]))
    want = []
    for k in range(7):  # more files than staging slots: the ring waits for the oldest
        sim.evolve_rk4_steps(2e-3, 1)
        want.append(reference_layout(sim.get_vertices(), f, sim.get_phi(), sim.get_psi()))
        sim.export_ply_async(tmp_path / f"mesh-{k}.ply")  # the next step is issued right after
    sim.export_wait()
    for k, w in enumerate(want):
        assert (tmp_path / f"mesh-{k}.ply").read_bytes() == w, k


def test_async_export_reports_write_errors(tmp_path):
    v, f = mesh.bubble(2, 1.0, (2.0, 0.0, 0.0))
    sim = ColocSim(v, f)
    sim.export_ply_async(tmp_path / "missing-dir" / "mesh.ply")
    with pytest.raises(Exception):
        sim.export_wait()
