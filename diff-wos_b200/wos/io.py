"""OBJ readers and writers for polylines and triangle meshes (reference:
wos/io.py:12-84, wos/scene.py:211-240, 463-475, wos/scene3d.py:116-144,
264-274): `v` vertex lines, `l` segment lines (2D), `f` face lines (3D) and
`c` per-vertex Dirichlet values, 1-based indices."""
from __future__ import annotations

import numpy as np


def _read(filename, elem: str, dim: int, flip_orientation: bool):
    """Vertices (float64, first `dim` coordinates), element indices (int64,
    0-based; for `l` lines the first two) and `c` values (float64), as the
    reference's readers return them (wos/io.py:20-38, :54-71)."""
    V, I, C = [], [], []
    with open(filename, "r") as f:
        for line in f:
            if line.startswith("v "):
                V.append([float(x) for x in line.split()[1:]][:dim])
            elif line.startswith(elem + " "):
                idx = [int(x.split("/")[0]) - 1 for x in line.split()[1:]]
                if flip_orientation:
                    idx = idx[::-1]
                I.append(idx[:2] if elem == "l" else idx)
            elif line.startswith("c "):
                C.append(float(line.split()[1]))
    return (np.asarray(V, np.float64).reshape(-1, dim), np.asarray(I, np.int64).reshape(-1, dim),
            np.asarray(C, np.float64))


def normalize_vertices(V):
    """Centre on the vertex mean and scale the farthest vertex to radius 1,
    in double precision, then round to float32 (wos/scene.py:232-237)."""
    V = np.asarray(V, np.float64)
    V = V - V.mean(0)
    return (V / np.linalg.norm(V, axis=1).max()).astype(np.float32)


def read_2d_obj(filename, flip_orientation=False):
    return _read(filename, "l", 2, flip_orientation)


def read_3d_obj(filename, flip_orientation=False):
    return _read(filename, "f", 3, flip_orientation)


def write_2d_obj(filename, vertices, indices, values=None):
    with open(filename, "w") as f:
        for v in vertices:
            f.write("v %f %f\n" % (v[0], v[1]))
        for i in indices:
            f.write("l %d %d\n" % (i[0] + 1, i[1] + 1))
        if values is not None:
            for c in values:
                f.write("c %f\n" % c)


def write_3d_obj(filename, vertices, indices, values=None):
    with open(filename, "w") as f:
        for v in vertices:
            f.write(f"v {v[0]} {v[1]} {v[2]}\n")
        for i in indices:
            f.write(f"f {i[0] + 1} {i[1] + 1} {i[2] + 1}\n")
        if values is not None:
            for c in values:
                f.write(f"c {c}\n")
