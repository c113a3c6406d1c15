"""Binary PLY meshes as the reference's drivers read them (Bem/Mesh/MeshIO.cpp import_ply): a vertex
element of float32 properties and a face element whose first property is a `list uchar int`.
Vertices are written with four float32 properties (x, y, z, value), the layout import_ply parses
as "4 floats"."""
import numpy as np


def write_ply(path, verts, trigs, values=None):
    verts = np.asarray(verts, dtype=np.float64)
    trigs = np.asarray(trigs, dtype=np.int32)
    vals = np.zeros(len(verts)) if values is None else np.asarray(values, dtype=np.float64)
    head = ("ply\nformat binary_little_endian 1.0\n"
            f"element vertex {len(verts)}\nproperty float x\nproperty float y\nproperty float z\n"
            "property float value\n"
            f"element face {len(trigs)}\nproperty list uchar int vertex_indices\nproperty uchar flags\n"
            "end_header\n")
    vrec = np.zeros(len(verts), dtype=[("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("v", "<f4")])
    vrec["x"], vrec["y"], vrec["z"], vrec["v"] = verts[:, 0], verts[:, 1], verts[:, 2], vals
    frec = np.zeros(len(trigs), dtype=[("n", "u1"), ("i", "<i4", (3,)), ("flag", "u1")])
    frec["n"] = 3
    frec["i"] = trigs
    with open(path, "wb") as fh:
        fh.write(head.encode("ascii"))
        fh.write(vrec.tobytes())
        fh.write(frec.tobytes())


def read_ply(path):
    """Binary little-endian PLY with float/double vertex properties and a `list uchar (u)int` face
    element (extra uchar face properties allowed).  Returns (verts (n,3), {name: values}, trigs)."""
    with open(path, "rb") as fh:
        data = fh.read()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    lines = data[:end].decode("ascii").splitlines()
    assert "format binary_little_endian 1.0" in lines
    elems, cur = [], None
    for ln in lines:
        w = ln.split()
        if w and w[0] == "element":
            cur = (w[1], int(w[2]), [])
            elems.append(cur)
        elif w and w[0] == "property":
            cur[2].append(w[1:])
    off = end
    out_v, out_f = None, None
    tmap = {"float": "<f4", "float32": "<f4", "double": "<f8", "float64": "<f8", "uchar": "u1", "uint8": "u1",
            "int": "<i4", "int32": "<i4", "uint": "<u4", "uint32": "<u4"}
    for name, count, props in elems:
        if name == "vertex":
            dt = np.dtype([(p[1], tmap[p[0]]) for p in props])
            out_v = np.frombuffer(data, dtype=dt, count=count, offset=off)
            off += dt.itemsize * count
        elif name == "face":
            lst = props[0]
            fields = [("n", tmap[lst[1]]), ("i", tmap[lst[2]], (3,))] + [(p[1], tmap[p[0]]) for p in props[1:]]
            dt = np.dtype(fields)
            out_f = np.frombuffer(data, dtype=dt, count=count, offset=off)
            assert np.all(out_f["n"] == 3)
            off += dt.itemsize * count
    verts = np.stack([out_v["x"], out_v["y"], out_v["z"]], 1).astype(np.float64)
    extra = {n: out_v[n].astype(np.float64) for n in out_v.dtype.names if n not in ("x", "y", "z")}
    return verts, extra, out_f["i"].astype(np.int64)
