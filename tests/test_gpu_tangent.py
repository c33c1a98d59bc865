"""Forward mode (derivative images) and the image-space boundary term.

The tangent of the per-point means along a direction of (vertices, values,
source parameters) is the same estimator as the adjoint, so for any point
weights w: sum_i w_i tangent_i = <adjoint(w), direction> (up to float32
storage).  A translated circle with values carried by its vertices moves its
solution rigidly, which gives the derivative in closed form.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_same_expectation, circle_scene, sphere_scene, star_scene

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("kind", ["star", "sphere"])
def test_tangent_equals_adjoint_along_direction(cuda, kind):
    import torch
    import wos
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    rng = np.random.default_rng(4)
    if kind == "star":
        V, F, g = star_scene(512)
        ns = NativeScene(V, F, g, 2, [1.0, -1.0, 0.3, 0.5, 1.0])
        P = rng.uniform(-0.4, 0.4, (300, 2)).astype(np.float32)
        s = WalkSettings(nwalks=16, nsteps=64, seed=21, include_source=True, use_IS_for_greens=True,
                         jitter=(0.01, 0.01, 0.0))
    else:
        V, F, g = sphere_scene(2)
        ns = NativeScene(V, F, g)
        P = rng.uniform(-0.4, 0.4, (200, 3)).astype(np.float32)
        s = WalkSettings(nwalks=16, nsteps=64, seed=21)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=kind == "star")
    dV = torch.tensor(rng.normal(size=V.shape).astype(np.float32), device="cuda")
    dg = torch.tensor(rng.normal(size=len(V)).astype(np.float32), device="cuda")
    ds = torch.tensor(rng.normal(size=5).astype(np.float32), device="cuda") if kind == "star" else None
    w = torch.tensor(rng.normal(size=len(P)).astype(np.float32), device="cuda")
    t = ns.solve_tangent(P, s, a, dV=dV, dg=dg, dsrc=ds, want_var=True)
    r = ns.solve_adjoint(P, s, a, loss_kind=0, target=w)
    assert np.array_equal(_np(t["mean"]), _np(r["mean"]))
    lhs = float((w.double() * t["tangent"]).sum())
    rhs = float((r["dV"].double() * dV.double()).sum() + (r["dg"].double() * dg.double()).sum())
    if ds is not None:
        rhs += float((r["dsrc"].double() * ds.double()).sum())
    assert abs(lhs - rhs) <= 1e-4 * (abs(rhs) + float((w.abs().double() * t["tangent"].abs()).sum())), (lhs, rhs)
    assert torch.isfinite(t["tangent_var"]).all()
    assert wos.device_status() == 0


def test_translated_circle_derivative_closed_form(cuda):
    """u = x^2 - y^2 on the unit circle, values carried by the vertices:
    translating by delta along x gives u = (x - delta)^2 - y^2, so the
    derivative of the solution is -2x."""
    import torch
    from wos import shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    V, F = shapes.circle(1024)
    g = (V[:, 0] ** 2 - V[:, 1] ** 2).astype(np.float32)
    ns = NativeScene(V, F, g)
    P = shapes.grid(48, -0.7, 0.7)
    P = np.ascontiguousarray(P[np.hypot(P[:, 0], P[:, 1]) < 0.7])
    s = WalkSettings(nwalks=256, nsteps=128, epsilon=1e-3, seed=5)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=False)
    e = np.zeros_like(V)
    e[:, 0] = 1.0
    t = ns.solve_tangent(P, s, a, dV=torch.tensor(e, device="cuda"), want_var=True)
    est, se = _np(t["tangent"]), np.sqrt(_np(t["tangent_var"]) / s.nwalks)
    exact = -2.0 * P[:, 0]
    # per point within the walks' standard errors (no added slack), and no
    # shared bias: the mean error within 4 standard errors of the mean
    assert_same_expectation(est, se, exact, np.zeros_like(exact), "translated circle")
    err = est - exact
    assert abs(err.mean()) < 4 * np.sqrt((se ** 2).sum()) / len(P), (err.mean(), np.sqrt((se ** 2).mean()))


def test_forward_ad_derivative_image(cuda):
    """torch forward-mode AD through walk_detector (the reference's renderD,
    diff_solve/runner.py:75-109): the walk term equals solve_tangent with the
    detector's jitter, and the boundary term's forward and reverse modes agree."""
    import torch
    import torch.autograd.forward_ad as fwAD
    import wos
    V, F, g = circle_scene(256)
    det = wos.Detector(vmin=(-1.2, -1.2), vmax=(1.2, 1.2), res=(40, 36))
    fwd = wos.WoSCUDA(nwalks=8, nsteps=64, epsilon=1e-3)
    bwd = wos.OursCUDA(nwalks=8, nsteps=64, epsilon=1e-3, epsilon2=1e-3)
    dirV = torch.zeros(V.shape, device="cuda")
    dirV[:, 0] = 1.0
    V0 = torch.tensor(V, device="cuda")
    with fwAD.dual_level():
        Vd = fwAD.make_dual(V0, dirV)
        scene = wos.Polyline(Vd, F, torch.tensor(g, device="cuda"))
        img = wos.CustomSolver(fwd, bwd).walk_detector(scene, det, seed=7)
        bimg = wos.WoSBoundary(nwalks=16).walk_detector(scene, det, seed=7)
        t_walk = fwAD.unpack_dual(img).tangent
        t_bnd = fwAD.unpack_dual(bimg).tangent
        b_primal = fwAD.unpack_dual(bimg).primal
    assert t_walk is not None and t_bnd is not None
    assert float(b_primal.abs().max()) == 0.0
    s = bwd.walk_settings(scene, 7, jitter=det.jitter())
    a = bwd.adjoint_settings(scene, True, False, False)
    ref = scene._native.solve_tangent(det.make_points(), s, a, dV=dirV)
    np.testing.assert_allclose(_np(t_walk), _np(ref["tangent"]).astype(np.float32), rtol=1e-6, atol=1e-6)
    # the boundary term lives on pixels the curve crosses
    nz = _np(t_bnd) != 0
    assert nz.any() and nz.sum() < 0.5 * nz.size
    # reverse mode of the same term
    Vr = torch.tensor(V, device="cuda", requires_grad=True)
    scene_r = wos.Polyline(Vr, F, torch.tensor(g, device="cuda"))
    wpix = torch.tensor(np.random.default_rng(2).normal(size=det.res[0] * det.res[1]).astype(np.float32),
                        device="cuda")
    (wos.WoSBoundary(nwalks=16).walk_detector(scene_r, det, seed=7) * wpix).sum().backward()
    lhs = float((wpix.double() * t_bnd.double()).sum())
    rhs = float((Vr.grad.double() * dirV.double()).sum())
    assert abs(lhs - rhs) <= 1e-4 * max(abs(rhs), 1e-6), (lhs, rhs)
    assert wos.device_status() == 0


def _odet(oracle, c):
    """The same wos_detector for the oracle."""
    return oracle.make_detector(tuple(c.vmin), tuple(c.vmax), tuple(c.res), c.axis_u, c.axis_v, c.slab_axis,
                                c.slab_center, c.slab_half_width, c.size, c.flags)


@pytest.mark.parametrize("kind,reference_pdf", [("star", False), ("star", True), ("sphere", False),
                                                ("sphere", True)])
def test_boundary_term_matches_oracle(cuda, oracle, kind, reference_pdf):
    """wos_boundary_term (k_boundary) against the oracle's restatement of
    WoSBoundary (wos/wos_boundary.py:11-31): same Philox samples, so the same
    primitives, pixels and contributions; the images and vertex gradients
    differ only by FP64 summation order.  With the reference's 3D pdf the 3D
    term is twice the default one; 2D is unchanged."""
    import torch
    import wos
    from wos.native import NativeScene
    rng = np.random.default_rng(12)
    if kind == "star":
        V, F, g = star_scene(512)
        det = wos.Detector(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(24, 20))
    else:
        V, F, g = sphere_scene(2)
        det = wos.Detector3D(vmin=(-1.2, -1.2), vmax=(1.2, 1.2), res=(24, 20), z=0.05)
    ns = NativeScene(V, F, g)
    os_ = oracle.OracleScene(V, F, g)
    wb = wos.WoSBoundary(nwalks=64, reference_area_pdf=reference_pdf)
    c = det.c(wb.flags())
    dV = rng.normal(size=V.shape).astype(np.float32)
    dLdI = rng.normal(size=det.res[0] * det.res[1]).astype(np.float32)
    img, gV = ns.boundary_term(c, 64, 9, dV_dir=torch.tensor(dV, device="cuda"),
                               dLdI=torch.tensor(dLdI, device="cuda"))
    oimg, ogV = os_.boundary_term(_odet(oracle, c), 64, 9, dV_dir=dV, dLdI=dLdI)
    assert np.count_nonzero(oimg) > 20
    np.testing.assert_allclose(_np(img), oimg, rtol=1e-9, atol=1e-12 * np.abs(oimg).max())
    np.testing.assert_allclose(_np(gV), ogV, rtol=1e-5, atol=1e-6 * np.abs(ogV).max())
    base, _ = ns.boundary_term(det.c(0), 64, 9, dV_dir=torch.tensor(dV, device="cuda"))
    factor = 2.0 if (reference_pdf and kind == "sphere") else 1.0
    # atomics add in a different order on every launch
    np.testing.assert_allclose(_np(img), factor * _np(base), rtol=1e-12, atol=1e-14 * np.abs(oimg).max())
    assert wos.device_status() == 0
