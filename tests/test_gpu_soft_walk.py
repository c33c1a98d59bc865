"""The soft-edge walk of Baseline / Baseline3D: values against the oracle,
forward-mode derivatives against central finite differences with common
random numbers, reverse mode against forward mode and finite differences, and
torch forward and reverse AD through Baseline."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("dim", [2, 3])
def test_soft_walk_matches_oracle(cuda, oracle, dim):
    from wos import shapes
    from wos.native import NativeScene, WalkSettings
    if dim == 2:
        V, F = shapes.star(512, 0.6, 0.2, 4)
        P = np.random.default_rng(1).uniform(-0.4, 0.4, (200, 2)).astype(np.float32)
    else:
        V, F = shapes.displaced_icosphere(2, 0.1, seed=2)
        P = np.random.default_rng(1).uniform(-0.4, 0.4, (150, 3)).astype(np.float32)
    g = np.cos(2 * V[:, 0] + V[:, 1]).astype(np.float32)
    ns, os_ = NativeScene(V, F, g), oracle.OracleScene(V, F, g)
    s = WalkSettings(nwalks=16, nsteps=48, epsilon=5e-3, seed=7, walk_offset=3)
    out = ns.soft_walk(P, s, want_var=True)
    ov = os_.soft_walk(P, oracle.make_params(16, 48, 5e-3, seed=7, walk_offset=3))
    om, _ = oracle.reduce(ov)
    np.testing.assert_allclose(_np(out["mean"]), om, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("dim", [2, 3])
def test_soft_walk_tangent_matches_finite_differences(cuda, dim):
    import torch
    from wos import shapes
    from wos.native import NativeScene, WalkSettings
    rng = np.random.default_rng(2)
    # coarse boundaries: a finite difference of step h crosses the kinks where
    # the nearest primitive changes about h / (primitive size) of the time
    if dim == 2:
        V, F = shapes.star(96, 0.6, 0.2, 4)
        P = rng.uniform(-0.35, 0.35, (256, 2)).astype(np.float32)
    else:
        V, F = shapes.displaced_icosphere(2, 0.1, seed=2)
        P = rng.uniform(-0.35, 0.35, (128, 3)).astype(np.float32)
    g = (V[:, 0] ** 2 - V[:, 1] ** 2 + 0.5 * V[:, 0]).astype(np.float32)
    dirV = rng.normal(size=V.shape).astype(np.float32) * 0.2
    dirV[:, 0] += 1.0
    dirg = rng.normal(size=len(V)).astype(np.float32)
    # Few steps: a soft walk that runs on creeps ever closer to the boundary,
    # where |sdf| has its kink and a finite difference of any fixed step h
    # stops resolving the derivative (the forward-mode tangent, like the
    # reference's AD, differentiates at the current distance).
    s = WalkSettings(nwalks=64, nsteps=8, epsilon=5e-2, seed=11)
    ns = NativeScene(V, F, g)
    t = ns.soft_walk(P, s, dV=torch.tensor(dirV, device="cuda"), dg=torch.tensor(dirg, device="cuda"),
                     want_tangent=True)
    h = 5e-5
    mp = NativeScene(V + h * dirV, F, g + h * dirg).soft_walk(P, s)["mean"]
    mm = NativeScene(V - h * dirV, F, g - h * dirg).soft_walk(P, s)["mean"]
    fd = _np((mp - mm) / (2 * h))
    tan = _np(t["tangent"])
    # the walk is a continuous function of the geometry; rare nearest-primitive
    # switches make single points noisy, so compare robustly
    err = np.abs(fd - tan)
    assert np.median(err) < 2e-2 * (np.median(np.abs(tan)) + 1e-3), (np.median(err), np.median(np.abs(tan)))
    assert abs(fd.mean() - tan.mean()) < 0.05 * (np.abs(tan).mean() + 1e-3)


def test_baseline_forward_ad_walk_detector(cuda):
    import torch
    import torch.autograd.forward_ad as fwAD
    import wos
    from wos import shapes
    V, F = shapes.circle(256)
    g = (V[:, 0] ** 2 - V[:, 1] ** 2).astype(np.float32)
    det = wos.Detector(vmin=(-0.7, -0.7), vmax=(0.7, 0.7), res=(20, 20))
    dirV = torch.zeros(V.shape, device="cuda")
    dirV[:, 0] = 1.0
    solver = wos.Baseline(nwalks=64, nsteps=64)
    with fwAD.dual_level():
        scene = wos.Polyline(fwAD.make_dual(torch.tensor(V, device="cuda"), dirV), F, torch.tensor(g, device="cuda"))
        img = solver.walk_detector(scene, det, seed=5)
        tan = fwAD.unpack_dual(img).tangent
        primal = fwAD.unpack_dual(img).primal
    s = solver.soft_settings(scene, 5, det.jitter())
    ref = scene._native.soft_walk(det.make_points(), s, dV=dirV, want_tangent=True)
    np.testing.assert_allclose(_np(primal), _np(ref["mean"]).astype(np.float32), rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(_np(tan), _np(ref["tangent"]).astype(np.float32), rtol=1e-6, atol=1e-6)
    # translation moves the (soft) solution rigidly: d/dt u = -2x inside
    P = _np(det.make_points())
    inside = np.hypot(P[:, 0], P[:, 1]) < 0.6
    assert abs(float(np.mean(_np(tan)[inside] + 2 * P[inside, 0]))) < 0.05
    # reverse mode through torch autograd is the native adjoint
    Vr = torch.tensor(V, device="cuda", requires_grad=True)
    gr = torch.tensor(g, device="cuda", requires_grad=True)
    scene_r = wos.Polyline(Vr, F, gr)
    w = torch.tensor(np.random.default_rng(3).normal(size=len(P)).astype(np.float32), device="cuda")
    (solver.walk(P, scene_r, seed=1) * w).sum().backward()
    dV, dg = scene_r._native.soft_walk_adjoint(P, solver.soft_settings(scene_r, 1), w)
    np.testing.assert_allclose(_np(Vr.grad), _np(dV), rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(_np(gr.grad), _np(dg), rtol=1e-6, atol=1e-7)



def _soft_case(dim, rng):
    from wos import shapes
    if dim == 2:
        V, F = shapes.star(96, 0.6, 0.2, 4)
        P = rng.uniform(-0.35, 0.35, (256, 2)).astype(np.float32)
    else:
        V, F = shapes.displaced_icosphere(2, 0.1, seed=2)
        P = rng.uniform(-0.35, 0.35, (128, 3)).astype(np.float32)
    g = (V[:, 0] ** 2 - V[:, 1] ** 2 + 0.5 * V[:, 0]).astype(np.float32)
    return V, F, g, P


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("use_bvh", [True, False])
def test_soft_walk_reverse_equals_forward(cuda, dim, use_bvh):
    """wos_soft_walk_adjoint is the transpose of the tangent recurrence: for
    point weights w and any direction, <adjoint(w), direction> =
    sum_i w_i tangent_i (FP64 sums of float32 walk terms)."""
    import torch
    import wos
    from wos.native import NativeScene, WalkSettings
    rng = np.random.default_rng(5)
    V, F, g, P = _soft_case(dim, rng)
    ns = NativeScene(V, F, g)
    s = WalkSettings(nwalks=32, nsteps=24, epsilon=2e-2, seed=13, use_bvh=use_bvh)
    dirV = torch.tensor(rng.normal(size=V.shape).astype(np.float32), device="cuda")
    dirg = torch.tensor(rng.normal(size=len(V)).astype(np.float32), device="cuda")
    w = torch.tensor(rng.normal(size=len(P)).astype(np.float32), device="cuda")
    t = ns.soft_walk(P, s, dV=dirV, dg=dirg, want_tangent=True)
    dV, dg = ns.soft_walk_adjoint(P, s, w)
    lhs = float((w.double() * t["tangent"]).sum())
    rhs = float((dV.double() * dirV.double()).sum() + (dg.double() * dirg.double()).sum())
    scale = float((w.abs().double() * t["tangent"].abs()).sum())
    assert abs(lhs - rhs) <= 1e-4 * scale, (lhs, rhs, scale)
    # each part alone
    tV = ns.soft_walk(P, s, dV=dirV, want_tangent=True)["tangent"]
    assert abs(float((w.double() * tV).sum()) - float((dV.double() * dirV.double()).sum())) <= 1e-4 * scale
    assert wos.device_status() == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_soft_walk_reverse_matches_finite_differences(cuda, dim):
    """The vertex gradient of L = sum_i w_i mean_i along a seeded direction
    against central finite differences with common random numbers, over 16
    seeds: within 2 standard errors."""
    import torch
    from wos.native import NativeScene, WalkSettings
    rng = np.random.default_rng(6)
    V, F, g, P = _soft_case(dim, rng)
    dirV = rng.normal(size=V.shape).astype(np.float32) * 0.2
    dirV[:, 0] += 1.0
    w = torch.tensor(rng.uniform(0.5, 1.5, len(P)).astype(np.float32), device="cuda")
    ns = NativeScene(V, F, g)
    h = 5e-5
    plus, minus = NativeScene(V + h * dirV, F, g), NativeScene(V - h * dirV, F, g)
    adj, fd = [], []
    for seed in range(16):
        s = WalkSettings(nwalks=64, nsteps=8, epsilon=5e-2, seed=100 + seed)
        dV, _ = ns.soft_walk_adjoint(P, s, w, want_dg=False)
        adj.append(float((dV.double() * torch.tensor(dirV, device="cuda").double()).sum()))
        lp = float((w.double() * plus.soft_walk(P, s)["mean"]).sum())
        lm = float((w.double() * minus.soft_walk(P, s)["mean"]).sum())
        fd.append((lp - lm) / (2 * h))
    adj, fd = np.array(adj), np.array(fd)
    se = np.sqrt(adj.var(ddof=1) / len(adj) + fd.var(ddof=1) / len(fd))
    z = (adj.mean() - fd.mean()) / se
    assert abs(z) < 2.0, (adj.mean(), fd.mean(), se)
