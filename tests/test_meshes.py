"""The reference's sample meshes (data/meshes, copied into tests/golden/meshes)
read by wos.io against what the reference's own readers return for them
(tests/golden/meshes_ref.npz, made by tests/golden/make_golden.py from
wos/io.py:20-38 read_2d_obj, :54-71 read_3d_obj and wos/scene.py:211-240
Polyline.from_obj), plus the CPU oracle's inside test on them: every mesh is
a closed, consistently oriented boundary whose interior the walks can use.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
MESH = GOLD / "meshes"
POLYLINES = ("wrench", "clover", "teapot")
TRIMESHES = ("bunny", "bunny2")


@pytest.fixture(scope="module")
def ref():
    return np.load(GOLD / "meshes_ref.npz")


@pytest.mark.parametrize("name", POLYLINES)
@pytest.mark.parametrize("flip", [False, True])
def test_read_2d_obj_matches_reference_reader(ref, name, flip):
    from wos import io
    V, F, c = io.read_2d_obj(MESH / f"{name}.obj", flip_orientation=flip)
    k = f"{name}_flip" if flip else name
    for got, want in ((V, ref[k + "_v"]), (F, ref[k + "_i"]), (c, ref[k + "_c"])):
        assert got.dtype == want.dtype
        np.testing.assert_array_equal(got, want.reshape(got.shape))


@pytest.mark.parametrize("name", TRIMESHES)
def test_read_3d_obj_matches_reference_reader(ref, name):
    from wos import io
    V, F, c = io.read_3d_obj(MESH / f"{name}.obj")
    for got, want in ((V, ref[name + "_v"]), (F, ref[name + "_i"]), (c, ref[name + "_c"])):
        assert got.dtype == want.dtype
        np.testing.assert_array_equal(got, want)
    # the bunny carries one `c` value per vertex
    assert len(c) == len(V) == 997 and len(F) == 1990


@pytest.mark.parametrize("name", POLYLINES)
def test_normalized_vertices_match_reference_from_obj(ref, name):
    from wos import io
    V, _, _ = io.read_2d_obj(MESH / f"{name}.obj")
    np.testing.assert_array_equal(io.normalize_vertices(V), ref[name + "_norm_v"])


def _grid(V, n, dim):
    lo, hi = V.min(0), V.max(0)
    axes = [np.linspace(lo[k], hi[k], n) for k in range(dim)]
    return np.stack([a.ravel() for a in np.meshgrid(*axes, indexing="ij")], 1).astype(np.float32)


@pytest.mark.parametrize("name,flip", [("wrench", True), ("clover", True), ("teapot", False)])
def test_reference_polylines_are_closed_and_ccw(oracle, name, flip):
    """Every vertex starts one segment and ends one, and the orientation the
    reference's scripts load them with (diff_solve/test_wrench.py:14-15 and
    ablations/test_clover.py:61-62 flip the wrench and the clover,
    diff_solve/test_teapot.py:16-17 keeps the teapot) is counter-clockwise,
    so the interior is sdf < 0."""
    from wos import io
    V, F, _ = io.read_2d_obj(MESH / f"{name}.obj", flip_orientation=flip)
    assert sorted(F[:, 0]) == list(range(len(V))) and sorted(F[:, 1]) == list(range(len(V)))
    a, b = V[F[:, 0]], V[F[:, 1]]
    assert 0.5 * np.sum(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]) > 0
    S = oracle.OracleScene(V.astype(np.float32), F.astype(np.int32), np.zeros(len(V), np.float32))
    P = _grid(V, 64, 2)
    out = S.closest(P)
    inside = out["inside"].astype(bool)
    assert 0.05 < inside.mean() < 0.95
    np.testing.assert_array_equal(inside, out["sdf"] < 0)


@pytest.mark.parametrize("name", TRIMESHES)
def test_reference_bunny_is_closed_and_outward(oracle, name):
    from wos import io
    V, F, _ = io.read_3d_obj(MESH / f"{name}.obj")
    # closed 2-manifold: every directed edge appears once and its reverse once
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    fwd = {tuple(x) for x in e}
    assert len(fwd) == len(e) and all((b, a) in fwd for a, b in fwd)
    p0, p1, p2 = (V[F[:, k]] for k in range(3))
    assert np.sum(np.einsum("ij,ij->i", p0, np.cross(p1 - p0, p2 - p0))) / 6 > 0  # positive volume
    S = oracle.OracleScene(V.astype(np.float32), F.astype(np.int32), np.zeros(len(V), np.float32))
    out = S.closest(_grid(V, 24, 3))
    inside = out["inside"].astype(bool)
    assert 0.05 < inside.mean() < 0.95
