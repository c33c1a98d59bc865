"""Edge cases: empty query sets on every compute entry point, degenerate and
open geometry against the oracle, and an empty item inside a batch."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _oparams(oracle, s):
    return oracle.make_params(s.nwalks, s.nsteps, s.epsilon, s.double_sided, s.prevent_fd_artifacts,
                              s.use_IS_for_greens, s.include_source, s.project_unterminated, s.use_bvh,
                              s.walk_offset, s.seed, s.jitter)


def test_empty_query_sets(cuda):
    import torch
    import wos
    from wos import shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    V, F = shapes.circle(64)
    ns = NativeScene(V, F, np.ones(len(V), np.float32))
    P = torch.empty((0, 2), device="cuda")
    s = WalkSettings(nwalks=4, nsteps=16)
    a = AdjointSettings(want_dV=True, want_dg=True)
    assert ns.solve(P, s).numel() == 0
    assert ns.values(P, s).shape == (0, 4)
    assert ns.closest(P)["prim"].numel() == 0
    out = ns.solve_adjoint(P, s, a, loss_kind=1)
    assert out["mean"].numel() == 0 and float(out["dV"].abs().sum()) == 0.0
    t = ns.solve_tangent(P, s, a, dV=torch.zeros((len(V), 2), device="cuda"))
    assert t["tangent"].numel() == 0
    assert wos.device_status() == 0


def test_zero_length_segment_matches_oracle(cuda, oracle):
    """A repeated vertex makes a zero-length segment (h = 0 there)."""
    from wos import shapes
    from wos.native import NativeScene, WalkSettings
    V, F = shapes.circle(128)
    V = np.insert(V, 10, V[10], axis=0)
    n = len(V)
    F = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1).astype(np.int32)
    g = (V[:, 0] ** 3 - 3 * V[:, 0] * V[:, 1] ** 2).astype(np.float32)
    ns, os_ = NativeScene(V, F, g), oracle.OracleScene(V, F, g)
    rng = np.random.default_rng(5)
    P = rng.uniform(-0.9, 0.9, (300, 2)).astype(np.float32)
    P[:5] = V[8:13] * 0.999
    s = WalkSettings(nwalks=8, nsteps=64, seed=3)
    vals, steps = ns.values(P, s, want_steps=True)
    ov, _, osteps = os_.walk_values(P, _oparams(oracle, s))
    assert np.array_equal(_np(vals), ov)
    assert np.array_equal(_np(steps), osteps)
    o = ns.closest(P)
    r = os_.closest(P, use_bvh=False)
    assert np.array_equal(_np(o["prim"]), r["prim"])


def test_open_polyline_double_sided_matches_oracle(cuda, oracle):
    """An open curve (no interior): double-sided walks terminate on either side."""
    from wos.native import NativeScene, WalkSettings
    t = np.linspace(-1.0, 1.0, 301)
    V = np.stack([t, 0.3 * np.sin(3 * t)], 1).astype(np.float32)
    F = np.stack([np.arange(300), np.arange(1, 301)], 1).astype(np.int32)
    g = np.cos(2 * V[:, 0]).astype(np.float32)
    ns, os_ = NativeScene(V, F, g), oracle.OracleScene(V, F, g)
    rng = np.random.default_rng(6)
    P = rng.uniform(-0.8, 0.8, (200, 2)).astype(np.float32)
    s = WalkSettings(nwalks=8, nsteps=128, seed=4, double_sided=True, project_unterminated=True)
    vals = ns.values(P, s)
    ov, _, _ = os_.walk_values(P, _oparams(oracle, s))
    assert np.array_equal(_np(vals), ov)


def test_batch_with_an_empty_item(cuda):
    import torch
    from wos import BatchItem, BatchPlan, shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    V, F = shapes.circle(256)
    ns = NativeScene(V, F, (V[:, 0] ** 2 - V[:, 1] ** 2).astype(np.float32))
    rng = np.random.default_rng(7)
    P1 = torch.tensor(rng.uniform(-0.5, 0.5, (300, 2)).astype(np.float32), device="cuda")
    P0 = torch.empty((0, 2), device="cuda")
    s = WalkSettings(nwalks=8, nsteps=64, seed=9)
    a = AdjointSettings(want_dV=True, want_dg=True)
    plan = BatchPlan([BatchItem(ns, P0, s, 1), BatchItem(ns, P1, s, 1)], a)
    plan.run(use_graph=True)
    o0, o1 = plan.outputs(0), plan.outputs(1)
    assert o0["mean"].numel() == 0 and float(o0["dV"].abs().sum()) == 0.0
    r = ns.solve_adjoint(P1, s, a, loss_kind=1)
    assert np.array_equal(_np(o1["mean"]), _np(r["mean"]))
    np.testing.assert_allclose(_np(o1["dV"]), _np(r["dV"]), rtol=1e-4, atol=1e-6 * float(r["dV"].abs().max()))
    plan.close()
