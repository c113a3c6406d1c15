"""Synthetic bubble meshes: frequency-nu geodesic icospheres and multi-bubble joins.

The vertex and face numbering reproduces the reference's input generator
(python_utils/icosphere/icosphere.py:34-68 ``icosphere``, :90-163 ``subdivide_mesh``,
:175-194 ``faces_template``, :197-224 ``vertex_ordering``, :227-245 ``inside_points``)
so that the unknowns of the dense system are numbered exactly as in the reference's
runs.  The layout is a format that has to match, so the enumeration order is the
same; the code below builds it from a (row, column) lattice per icosahedron face.

Numbering (per face f with corners A, B, C, lattice row i = 0..nu, column j = 0..i):
  * the 12 icosahedron corners come first;
  * then nu-1 points per icosahedron edge, edges sorted by (min, max) corner, each edge
    enumerated from its smaller corner (weight (nu-1-k)/nu on it, k = 0..nu-2);
  * then (nu-1)(nu-2)/2 interior points per face, row by row, left to right.
Faces: nu^2 per icosahedron face, row by row; in row i first the pairs
((i,j),(i+1,j),(i+1,j+1)) and ((i,j),(i+1,j+1),(i,j+1)) for j < i, then the last
((i,i),(i+1,i),(i+1,i+1)).

Floating point: edge points are w_hi*P + w_lo*Q and interior points are the same blend of
two (unnormalised) edge points, then every point is divided by sqrt((x*x+y*y)+z*z).  These
are the reference's element-wise operations, so the arrays are bit-identical.
"""
from __future__ import annotations

import numpy as np

_ICO_FACES = np.array([
    [0, 5, 1], [0, 3, 5], [0, 2, 3], [0, 4, 2], [0, 1, 4],
    [1, 5, 8], [5, 3, 10], [3, 2, 7], [2, 4, 11], [4, 1, 9],
    [7, 11, 6], [11, 9, 6], [9, 8, 6], [8, 10, 6], [10, 7, 6],
    [2, 11, 7], [4, 9, 11], [1, 8, 9], [5, 10, 8], [3, 7, 10]], dtype=np.int64)


def _icosahedron():
    g = (1 + np.sqrt(5)) / 2
    top = np.array([[0, 1, g], [0, -1, g], [1, g, 0],
                    [-1, g, 0], [g, 0, 1], [-g, 0, 1]]) / np.sqrt(1 + g ** 2)
    return np.concatenate([top, -top], axis=0), _ICO_FACES.copy()


def icosphere(nu: int):
    """Unit geodesic sphere: 10*nu^2+2 vertices (float64, shape (N,3)) and 20*nu^2
    outward-oriented triangles (int64, shape (M,3))."""
    nu = int(nu)
    if nu < 1:
        raise ValueError("subdivision frequency must be >= 1")
    verts, faces = _icosahedron()
    if nu == 1:
        return verts, faces
    V, F = verts.shape[0], faces.shape[0]
    pairs = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [0, 2]]])
    edges = np.unique(np.sort(pairs, axis=1), axis=0)
    E = edges.shape[0]
    edge_id = {(int(a), int(b)): e for e, (a, b) in enumerate(edges)}
    n_edge_pts = nu - 1
    n_face_pts = (nu - 1) * (nu - 2) // 2
    out = np.empty((V + E * n_edge_pts + F * n_face_pts, 3))
    out[:V] = verts
    w = np.arange(1, nu) / nu
    k = np.arange(n_edge_pts)
    for e in range(E):
        p, q = verts[edges[e, 0]], verts[edges[e, 1]]
        out[V + e * n_edge_pts + k] = w[::-1][k, None] * p + w[k, None] * q

    def edge_points(a: int, b: int) -> np.ndarray:
        """Indices of the points on edge a->b, enumerated starting next to a."""
        lo, hi = (a, b) if a < b else (b, a)
        e = edge_id[(lo, hi)]
        idx = V + e * n_edge_pts + np.arange(n_edge_pts)
        # the reference keys the direction by the sign of the edge id, so edge 0 is
        # never flipped; its two faces only use it in the a<b direction
        flip = (a > b) and e != 0
        return idx[::-1] if flip else idx

    # lattice templates, identical for every face
    rows = [(i, j) for i in range(nu + 1) for j in range(i + 1)]
    tri_ij = []
    for i in range(nu):
        for j in range(i):
            tri_ij.append(((i, j), (i + 1, j), (i + 1, j + 1)))
            tri_ij.append(((i, j), (i + 1, j + 1), (i, j + 1)))
        tri_ij.append(((i, i), (i + 1, i), (i + 1, i + 1)))
    out_faces = np.empty((F * nu * nu, 3), dtype=np.int64)
    base_face_pts = V + E * n_edge_pts
    for f in range(F):
        A, B, C = (int(t) for t in faces[f])
        AB, AC, BC = edge_points(A, B), edge_points(A, C), edge_points(B, C)
        interior0 = base_face_pts + f * n_face_pts
        lut = {}
        t = 0
        for (i, j) in rows:
            if i == 0:
                lut[(i, j)] = A
            elif i == nu:
                lut[(i, j)] = B if j == 0 else (C if j == nu else int(BC[j - 1]))
            elif j == 0:
                lut[(i, j)] = int(AB[i - 1])
            elif j == i:
                lut[(i, j)] = int(AC[i - 1])
            else:
                lut[(i, j)] = interior0 + t
                t += 1
        # interior point geometry: blend of the edge points of the same row
        for i in range(2, nu):
            cnt = i - 1
            wi = np.arange(1, cnt + 1) / (cnt + 1)
            pa, pc = out[AB[i - 1]], out[AC[i - 1]]
            for kk in range(cnt):
                out[lut[(i, kk + 1)]] = wi[cnt - 1 - kk] * pa + wi[kk] * pc
        out_faces[f * nu * nu:(f + 1) * nu * nu] = [[lut[a], lut[b], lut[c]] for (a, b, c) in tri_ij]
    nrm = np.sqrt((out[:, 0] * out[:, 0] + out[:, 1] * out[:, 1]) + out[:, 2] * out[:, 2])
    out = out / nrm[:, None]
    return out, out_faces


def join(parts):
    """Concatenate (verts, faces) pairs as the reference's join_meshes does
    (Bem/Mesh/Mesh.cpp:356-362, Mesh::add :12-23): vertices appended in order,
    triangle indices offset by the running vertex count."""
    vs, fs, off = [], [], 0
    for v, f in parts:
        vs.append(np.asarray(v, dtype=np.float64))
        fs.append(np.asarray(f, dtype=np.int64) + off)
        off += len(v)
    return np.concatenate(vs, axis=0), np.concatenate(fs, axis=0)


def bubble(nu: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """Icosphere scaled by ``radius`` then translated by ``center``
    (Mesh::scale then Mesh::translate, Bem/Mesh/Mesh.cpp:24-27,47-50)."""
    v, f = icosphere(nu)
    v = v * float(radius)
    v = v + np.asarray(center, dtype=np.float64)[None, :]
    return v, f


def signed_volume(verts, faces) -> float:
    """Sum of (a x b).c / 6 over triangles (Bem/Mesh/Mesh.cpp:206-218)."""
    a, b, c = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    return float(np.sum(np.einsum("ij,ij->i", np.cross(a, b), c)) / 6.0)


def wall_cap(nu: int, radius: float = 1.0):
    """Hemisphere of ``radius`` sitting on the wall x = 0 (centre at the origin, x >= 0): the four
    octants of a geodesic octahedron sphere with x > 0, each face cut into nu^2 triangles, the
    vertices normalised to the sphere.  The boundary loop (4*nu vertices) lies exactly on x = 0, the
    contact line of a pinned bubble (the reference's ColocSimPin meshes).  Outward orientation."""
    if nu < 1:
        raise ValueError("nu >= 1")
    X, Y, Z = np.eye(3)
    corners = {"x": X, "y": Y, "z": Z, "-y": -Y, "-z": -Z}
    faces = [("x", "y", "z"), ("x", "z", "-y"), ("x", "-y", "-z"), ("x", "-z", "y")]
    index, pts, tris = {}, [], []

    def vid(key_weights):
        key = tuple(sorted((c, w) for c, w in key_weights if w))
        if key not in index:
            p = sum(w * corners[c] for c, w in key) / nu
            index[key] = len(pts)
            pts.append(p)
        return index[key]

    for a, b, c in faces:
        lat = {(i, j): vid(((a, nu - i), (b, i - j), (c, j))) for i in range(nu + 1) for j in range(i + 1)}
        for i in range(nu):
            for j in range(i + 1):
                tris.append((lat[(i, j)], lat[(i + 1, j)], lat[(i + 1, j + 1)]))
                if j < i:
                    tris.append((lat[(i, j)], lat[(i + 1, j + 1)], lat[(i, j + 1)]))
    v = np.array(pts, dtype=np.float64)
    v = v / np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])[:, None] * float(radius)
    return v, np.array(tris, dtype=np.int64)
