"""The CUDA path on the reference's own sample meshes (data/meshes, copied into
tests/golden/meshes) against the CPU oracle: the wrench as
diff_solve/test_wrench.py:12-17 poses it (flipped, scaled by 1.2, shifted by
(0.1, -0.1)), the clover as ablations/test_clover.py:61-62 loads it, and the
bunny of diff_solve/test_bunny.py:23-24, each with its own `c` values
(zeros for the clover, which has none).  Nearest primitives, distances and
per-walk values are compared bit for bit, adjoint gradients to 1e-4."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MESH = Path(__file__).resolve().parent / "golden" / "meshes"
GRAD_RTOL = 1e-4


def _np(t):
    return t.detach().cpu().numpy()


def _mesh(name):
    from wos import io
    if name == "wrench":
        V, F, g = io.read_2d_obj(MESH / "wrench.obj", flip_orientation=True)
        V = V * 1.2 + np.array([0.1, -0.1])
    elif name == "clover":
        V, F, g = io.read_2d_obj(MESH / "clover.obj", flip_orientation=True)
        g = np.zeros(len(V))
    else:
        V, F, g = io.read_3d_obj(MESH / f"{name}.obj")
    return V.astype(np.float32), F.astype(np.int32), g.astype(np.float32)


def _interior(oracle, V, F, g, n):
    S = oracle.OracleScene(V, F, g)
    lo, hi = V.min(0), V.max(0)
    rng = np.random.default_rng(7)
    P = rng.uniform(lo, hi, (8 * n, V.shape[1])).astype(np.float32)
    return P[S.closest(P)["inside"].astype(bool)][:n], S


def _oparams(oracle, s):
    return oracle.make_params(s.nwalks, s.nsteps, s.epsilon, s.double_sided, s.prevent_fd_artifacts,
                              s.use_IS_for_greens, s.include_source, s.project_unterminated, s.use_bvh,
                              s.walk_offset, s.seed, s.jitter)


@pytest.mark.parametrize("name", ["wrench", "clover", "bunny", "bunny2"])
def test_reference_mesh_queries_and_walks_bit_exact(cuda, oracle, name):
    from wos.native import NativeScene, WalkSettings
    V, F, g = _mesh(name)
    P, S = _interior(oracle, V, F, g, 600 if V.shape[1] == 2 else 300)
    assert len(P) > 100
    ns = NativeScene(V, F, g)
    Q = np.concatenate([P, V[:64] + 0.01, V[:16]]).astype(np.float32)
    for use_bvh in (True, False):
        o = ns.closest(Q, use_bvh)
        r = S.closest(Q, use_bvh=False)
        assert np.array_equal(_np(o["prim"]), r["prim"])
        assert np.array_equal(_np(o["dist"]), r["dist"])
        assert np.array_equal(_np(o["inside"]), r["inside"])
    s = WalkSettings(nwalks=4, nsteps=128, epsilon=1e-3, seed=31)
    vals, steps = ns.values(P, s, want_steps=True)
    ov, _, osteps = S.walk_values(P, _oparams(oracle, s))
    assert np.array_equal(_np(vals), ov)
    assert np.array_equal(_np(steps), osteps)
    import wos
    assert wos.device_status() == 0


@pytest.mark.parametrize("name", ["wrench", "bunny"])
def test_reference_mesh_adjoint_matches_oracle(cuda, oracle, name):
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    V, F, g = _mesh(name)
    P, S = _interior(oracle, V, F, g, 120 if V.shape[1] == 2 else 80)
    ns = NativeScene(V, F, g)
    rng = np.random.default_rng(3)
    dLdu = rng.normal(size=len(P)).astype(np.float32)
    s = WalkSettings(nwalks=8, nsteps=128, epsilon=1e-3, seed=5)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True)
    dV, dg, _ = ns.adjoint(P, s, a, dLdu)
    odV, odg, _ = S.adjoint(P, _oparams(oracle, s), oracle.make_adj(1e-3, 0.1, True, False, 1e-3, True, True, False),
                            dLdu)
    np.testing.assert_allclose(_np(dV), odV, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odV).max())
    np.testing.assert_allclose(_np(dg), odg, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odg).max())
