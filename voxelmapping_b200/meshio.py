"""Mesh export: the triangles of VoxelMapping.Polygonize (9 floats per
triangle for the vertices and for the normals, world metres) as a binary
little-endian PLY file with per-vertex normals. The reference hands the
buffers to its viewer (example/pangolin_display_3d.cpp) and writes no file."""
import numpy as np


def write_ply(path, verts, norms=None):
    """verts, norms: (n, 9) float32 as returned by Polygonize. Each triangle
    becomes three vertices and one face (vertices are not merged)."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    n_tri = v.shape[0] // 3
    cols = [("x", "<f4"), ("y", "<f4"), ("z", "<f4")]
    if norms is not None:
        cols += [("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4")]
    vert = np.empty(v.shape[0], dtype=cols)
    vert["x"], vert["y"], vert["z"] = v[:, 0], v[:, 1], v[:, 2]
    if norms is not None:
        nm = np.ascontiguousarray(norms, np.float32).reshape(-1, 3)
        vert["nx"], vert["ny"], vert["nz"] = nm[:, 0], nm[:, 1], nm[:, 2]
    face = np.empty(n_tri, dtype=[("n", "u1"), ("i", "<i4", 3)])
    face["n"] = 3
    face["i"] = np.arange(3 * n_tri, dtype=np.int32).reshape(-1, 3)
    header = ["ply", "format binary_little_endian 1.0", "element vertex %d" % v.shape[0]]
    header += ["property float %s" % c for c, _ in cols]
    header += ["element face %d" % n_tri, "property list uchar int vertex_indices", "end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n").encode("ascii"))
        f.write(vert.tobytes())
        f.write(face.tobytes())


def read_ply(path):
    """(verts (n, 9), norms (n, 9) or None) of a file written by write_ply."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    header = data[:end].decode("ascii").splitlines()
    nv = int(next(h for h in header if h.startswith("element vertex")).split()[2])
    nf = int(next(h for h in header if h.startswith("element face")).split()[2])
    props = [h.split()[2] for h in header if h.startswith("property float")]
    vert = np.frombuffer(data, dtype=[(p, "<f4") for p in props], count=nv, offset=end)
    face = np.frombuffer(data, dtype=[("n", "u1"), ("i", "<i4", 3)], count=nf, offset=end + vert.nbytes)
    idx = face["i"].reshape(-1)
    xyz = np.stack([vert["x"], vert["y"], vert["z"]], 1)[idx].reshape(-1, 9)
    nrm = np.stack([vert["nx"], vert["ny"], vert["nz"]], 1)[idx].reshape(-1, 9) if "nx" in props else None
    return xyz, nrm
