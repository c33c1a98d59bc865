"""OBJ readers and writers for polylines and triangle meshes (reference:
wos/io.py:12-84, wos/scene.py:211-240, 463-475, wos/scene3d.py:116-144,
264-274): `v` vertex lines, `l` segment lines (2D), `f` face lines (3D) and
`c` per-vertex Dirichlet values, 1-based indices."""
from __future__ import annotations

import numpy as np


def _read(filename, elem: str, dim: int, flip_orientation: bool):
    V, I, C = [], [], []
    with open(filename, "r") as f:
        for line in f:
            line = line.strip()
            if line.startswith("v "):
                V.append([float(x) for x in line[2:].split()][:dim])
            elif line.startswith(elem + " "):
                idx = [int(x.split("/")[0]) - 1 for x in line[2:].split()]
                if flip_orientation:
                    idx = idx[::-1]
                I.append(idx)
            elif line.startswith("c "):
                C.append(float(line[2:].split()[0]))
    return np.asarray(V, np.float32).reshape(-1, dim), np.asarray(I, np.int32).reshape(-1, dim), np.asarray(
        C, np.float32)


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
