"""CUDA path against the CPU oracle on the same seeded inputs.

Integer and index results (nearest primitive, validity, step counts) and the
per-walk float results are compared bit for bit: both sides evaluate the same
float32 operation sequence (explicit fmaf, IEEE sqrt/div, the same
polynomial sin/cos/log, Philox counters), so any difference is a bug.  Sums
over many walks (means, adjoint gradients) are compared with a stated
relative tolerance because their summation order differs.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import circle_scene, sphere_scene, star_scene

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-4  # float64 accumulation in a different order, stored as float32


def _scenes(oracle, V, F, g, source_type=0, source_params=None):
    from wos.native import NativeScene
    return NativeScene(V, F, g, source_type, source_params), oracle.OracleScene(V, F, g, source_type, source_params)


def _np(t):
    return t.detach().cpu().numpy()


def _pts2(n, seed=0, lo=-0.95, hi=0.95):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, 2)).astype(np.float32)


def _pts3(n, seed=0, lo=-1.1, hi=1.1):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, 3)).astype(np.float32)


def _settings(**kw):
    from wos.native import WalkSettings
    return WalkSettings(**kw)


def _oparams(oracle, s):
    return oracle.make_params(s.nwalks, s.nsteps, s.epsilon, s.double_sided, s.prevent_fd_artifacts,
                              s.use_IS_for_greens, s.include_source, s.project_unterminated, s.use_bvh,
                              s.walk_offset, s.seed, s.jitter)


# ---------------------------------------------------------------- scene build
@pytest.mark.parametrize("kind", ["circle", "star", "sphere"])
def test_normals_and_aabb_match_oracle(cuda, oracle, kind):
    V, F, g = {"circle": circle_scene, "star": star_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    assert np.array_equal(_np(ns.normals()), os_.normals())
    lo, hi = os_.aabb()
    info = ns.info()
    d = V.shape[1]
    assert np.array_equal(np.array(info.aabb_min[:d], np.float32), lo)
    assert np.array_equal(np.array(info.aabb_max[:d], np.float32), hi)
    assert info.n_nodes == F.shape[0] - 1
    assert 0 < info.bvh_depth <= 64


# ---------------------------------------------------------------- queries
@pytest.mark.parametrize("kind", ["circle", "star", "sphere"])
@pytest.mark.parametrize("use_bvh", [True, False])
def test_closest_point_bit_exact(cuda, oracle, kind, use_bvh):
    V, F, g = {"circle": circle_scene, "star": star_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(4000, 1) if V.shape[1] == 2 else _pts3(3000, 1)
    # add exact vertices, edge midpoints and far-away points (ties, zero distance)
    extra = np.concatenate([V[:50], 0.5 * (V[F[:50, 0]] + V[F[:50, 1]]), V[:20] * 7.0]).astype(np.float32)
    P = np.concatenate([P, extra])
    o = ns.closest(P, use_bvh)
    r = os_.closest(P, use_bvh=False)  # oracle brute force is the reference answer
    assert np.array_equal(_np(o["prim"]), r["prim"])
    assert np.array_equal(_np(o["dist"]), r["dist"])
    assert np.array_equal(_np(o["tuv"]), r["tuv"])
    assert np.array_equal(_np(o["pt"]), r["pt"])
    assert np.array_equal(_np(o["n"]), r["n"])
    assert np.array_equal(_np(o["sdf"]), r["sdf"])
    assert np.array_equal(_np(o["inside"]), r["inside"])
    assert np.array_equal(_np(ns.sdf(P, use_bvh)), r["sdf"])  # wos_sdf


def test_bvh_equals_brute_force_ties(cuda, oracle):
    # a square with duplicated collinear segments: many exact distance ties
    V = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1], [0, -1], [0, 1]], np.float32)
    F = np.array([[0, 4], [4, 1], [1, 2], [2, 5], [5, 3], [3, 0], [0, 4], [2, 5]], np.int32)
    g = np.zeros(6, np.float32)
    ns, os_ = _scenes(oracle, V, F, g)
    P = np.stack(np.meshgrid(np.linspace(-1.5, 1.5, 61), np.linspace(-1.5, 1.5, 61)), -1).reshape(-1, 2)
    P = P.astype(np.float32)
    a = _np(ns.closest(P, True)["prim"])
    b = _np(ns.closest(P, False)["prim"])
    assert np.array_equal(a, b)
    assert np.array_equal(a, os_.closest(P, use_bvh=False)["prim"])


@pytest.mark.parametrize("kind", ["circle", "sphere"])
def test_inscribed_ball_bit_exact(cuda, oracle, kind):
    V, F, g = {"circle": circle_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(2000, 2, -0.8, 0.8) if V.shape[1] == 2 else _pts3(2000, 2, -0.7, 0.7)
    r = os_.closest(P)
    valid = (np.arange(len(P)) % 7 != 0).astype(np.uint8)
    R_gpu = _np(ns.inscribed_ball(valid, r["pt"], r["n"], 1e-3, True))
    R_orc = os_.inscribed_ball(valid, r["pt"], r["n"], 1e-3)
    assert np.array_equal(R_gpu, R_orc)
    assert (R_gpu[valid == 0] == 0).all()


# ---------------------------------------------------------------- walks
WALK_CASES = [
    ("circle", dict()),
    ("circle", dict(nsteps=4)),
    ("circle", dict(project_unterminated=True, nsteps=6)),
    ("circle", dict(double_sided=True)),
    ("circle", dict(prevent_fd_artifacts=True)),
    ("circle", dict(use_bvh=False)),
    ("star", dict(epsilon=1e-4, nsteps=64)),
    ("sphere", dict()),
    ("sphere", dict(use_bvh=False, nsteps=8)),
    ("sphere", dict(double_sided=True, nsteps=16)),
    ("circle", dict(jitter=(0.02, 0.03, 0.0))),
    ("sphere", dict(jitter=(0.02, 0.0, 0.05))),
]


@pytest.mark.parametrize("kind,kw", WALK_CASES)
def test_walk_values_bit_exact(cuda, oracle, kind, kw):
    V, F, g = {"circle": circle_scene, "star": star_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(300, 3) if V.shape[1] == 2 else _pts3(200, 3)
    s = _settings(nwalks=16, nsteps=kw.pop("nsteps", 32), seed=1234, walk_offset=5, **kw)
    vals, steps = ns.values(P, s, want_steps=True)
    ov, ovalid, osteps = os_.walk_values(P, _oparams(oracle, s))
    assert np.array_equal(_np(steps), osteps)
    assert np.array_equal(_np(vals), ov)
    plain = ns.values(P, s, plain=True)
    assert np.array_equal(_np(plain), ov)


@pytest.mark.parametrize("use_IS", [False, True])
@pytest.mark.parametrize("src", [(2, [0.0, 0.0, 0.0, 0.0, 1.0]), (2, [3.0, -2.0, 0.5, 1.5, 0.25]),
                                 (1, [0.1, -0.2, 0.3, 0.25, 2.0])])
def test_walk_with_source_bit_exact(cuda, oracle, use_IS, src):
    V, F, g = star_scene(1024)
    ns, os_ = _scenes(oracle, V, F, g, src[0], src[1])
    P = _pts2(400, 4, -0.5, 0.5)
    s = _settings(nwalks=8, nsteps=64, seed=99, include_source=True, use_IS_for_greens=use_IS)
    vals = ns.values(P, s)
    ov, _, _ = os_.walk_values(P, _oparams(oracle, s))
    assert np.array_equal(_np(vals), ov)
    rec = ns.records(P, s)
    orec = os_.walk_records(P, _oparams(oracle, s))
    assert np.array_equal(_np(rec["contrib"]), orec["contrib"])


@pytest.mark.parametrize("kind", ["circle", "sphere"])
def test_walk_records_bit_exact(cuda, oracle, kind):
    V, F, g = {"circle": circle_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(1000, 5) if V.shape[1] == 2 else _pts3(800, 5)
    s = _settings(nwalks=1, nsteps=64, seed=7, walk_offset=3)
    rec = ns.records(P, s)
    orec = os_.walk_records(P, _oparams(oracle, s))
    for k in ("valid", "pt", "n", "tuv", "prim"):
        assert np.array_equal(_np(rec[k]), orec[k]), k


def test_solve_mean_and_variance(cuda, oracle):
    V, F, g = circle_scene()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(500, 6, -0.6, 0.6)
    s = _settings(nwalks=100, nsteps=64, seed=3)
    mean, var = ns.solve(P, s, want_var=True)
    ov, _, _ = os_.walk_values(P, _oparams(oracle, s))
    om, ovar = oracle.reduce(ov)
    np.testing.assert_allclose(_np(mean), om, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(_np(var), ovar, rtol=1e-10, atol=1e-14)


def test_results_independent_of_launch_shape(cuda, oracle):
    import wos
    V, F, g = star_scene(2048)
    ns, _ = _scenes(oracle, V, F, g)
    P = _pts2(2000, 8, -0.5, 0.5)
    s = _settings(nwalks=32, nsteps=64, seed=11)
    base = _np(ns.values(P, s))
    old = wos.get_launch_config(2)
    try:
        for bt, chunk, nodes in [(64, 1, 0), (128, 7, 16), (512, 256, 4000)]:
            wos.set_launch_config(2, block_threads=bt, chunk=chunk, smem_nodes=nodes)
            assert np.array_equal(_np(ns.values(P, s)), base)
    finally:
        wos.set_launch_config(2, old.block_threads, old.blocks_per_sm, old.chunk, old.smem_nodes)


# ---------------------------------------------------------------- gradients
@pytest.mark.parametrize("kind", ["circle", "sphere"])
def test_normal_derivative_bit_exact(cuda, oracle, kind):
    from wos.native import AdjointSettings
    V, F, g = {"circle": circle_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(600, 9, -0.7, 0.7) if V.shape[1] == 2 else _pts3(400, 9, -0.6, 0.6)
    s = _settings(nwalks=1, nsteps=64, seed=21)
    orec = os_.walk_records(P, _oparams(oracle, s))
    a = AdjointSettings(epsilon2=5e-4, clamping=0.1)
    nd = _np(ns.normal_derivative(orec, s, a))
    ond = os_.normal_derivative(orec, _oparams(oracle, s), oracle.make_adj(5e-4, 0.1))
    assert np.array_equal(nd, ond)


@pytest.mark.parametrize("kind,src", [("circle", None), ("star", (2, [1.0, -1.0, 0.3, 0.5, 1.0])),
                                      ("sphere", None)])
def test_adjoint_matches_oracle(cuda, oracle, kind, src):
    from wos.native import AdjointSettings
    if kind == "star":
        V, F, g = star_scene(512)
        ns, os_ = _scenes(oracle, V, F, g, *src)
    else:
        V, F, g = {"circle": lambda: circle_scene(256), "sphere": lambda: sphere_scene(2)}[kind]()
        ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(200, 10, -0.5, 0.5) if V.shape[1] == 2 else _pts3(150, 10, -0.5, 0.5)
    rng = np.random.default_rng(10)
    dLdu = rng.normal(size=len(P)).astype(np.float32)
    s = _settings(nwalks=8, nsteps=64, seed=5, include_source=src is not None)
    a = AdjointSettings(epsilon2=5e-4, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=src is not None)
    dV, dg, ds = ns.adjoint(P, s, a, dLdu)
    oa = oracle.make_adj(5e-4, 0.1, True, True, 1e-3, True, True, src is not None)
    odV, odg, ods = os_.adjoint(P, _oparams(oracle, s), oa, dLdu)
    scale = np.abs(odV).max()
    np.testing.assert_allclose(_np(dV), odV, rtol=GRAD_RTOL, atol=GRAD_RTOL * scale)
    np.testing.assert_allclose(_np(dg), odg, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odg).max())
    if src is not None:
        np.testing.assert_allclose(_np(ds), ods, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(ods).max())


def test_device_status_clean(cuda):
    import wos
    assert wos.device_status(reset=False) == 0


# ---------------------------------------------------------------- fused path
@pytest.mark.parametrize("kind,src,jitter", [("circle", None, None), ("star", (2, [0.0, 0.0, 0.0, 0.0, 1.0]), None),
                                             ("sphere", None, None), ("circle", None, (0.05, 0.04, 0.0)),
                                             ("sphere", None, (0.05, 0.04, 0.0))])
def test_fused_solve_adjoint_matches_oracle(cuda, oracle, kind, src, jitter):
    from wos.native import AdjointSettings
    if kind == "star":
        V, F, g = star_scene(512)
        ns, os_ = _scenes(oracle, V, F, g, *src)
    else:
        V, F, g = {"circle": lambda: circle_scene(256), "sphere": lambda: sphere_scene(2)}[kind]()
        ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(150, 12, -0.5, 0.5) if V.shape[1] == 2 else _pts3(120, 12, -0.5, 0.5)
    s = _settings(nwalks=8, nsteps=64, seed=77, include_source=src is not None, use_IS_for_greens=src is not None,
                  jitter=jitter or (0.0, 0.0, 0.0))
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=src is not None)
    out = ns.solve_adjoint(P, s, a, loss_kind=1)
    ov, _, _ = os_.walk_values(P, _oparams(oracle, s))
    om, _ = oracle.reduce(ov)
    np.testing.assert_allclose(_np(out["mean"]), om, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(_np(out["loss"])[0], (om ** 2).mean(), rtol=1e-10)
    dLdu = (2.0 * _np(out["mean"]) / len(P)).astype(np.float32)
    oa = oracle.make_adj(1e-3, 0.1, True, True, 1e-3, True, True, src is not None)
    odV, odg, ods = os_.adjoint(P, _oparams(oracle, s), oa, dLdu)
    np.testing.assert_allclose(_np(out["dV"]), odV, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odV).max())
    np.testing.assert_allclose(_np(out["dg"]), odg, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odg).max())
    if src is not None:
        np.testing.assert_allclose(_np(out["dsrc"]), ods, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(ods).max())


def test_records_adjoint_equals_recomputed(cuda, oracle):
    from wos.native import AdjointSettings
    V, F, g = star_scene(1024)
    ns, _ = _scenes(oracle, V, F, g, 2, [1.0, 2.0, 0.0, 0.5, 1.0])
    P = _pts2(300, 13, -0.5, 0.5)
    s = _settings(nwalks=16, nsteps=64, seed=5, include_source=True, use_IS_for_greens=True)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=True)
    mean, _, rec, dc = ns.solve_records(P, s, want_dcontrib=True)
    assert np.array_equal(_np(mean), _np(ns.solve(P, s)))
    dLdu = (2.0 / len(P)) * mean.float()
    r1 = ns.adjoint_records(P, s, a, dLdu, rec, dc)
    r2 = ns.adjoint(P, s, a, dLdu)
    for x, y in zip(r1, r2):
        np.testing.assert_allclose(_np(x), _np(y), rtol=1e-5, atol=1e-6 * np.abs(_np(y)).max())


def test_autograd_custom_solver_matches_native(cuda, oracle):
    import torch
    import wos
    from wos.native import AdjointSettings
    V, F, g = star_scene(512)
    src = [0.0, 0.0, 0.0, 0.0, 1.0]
    P = _pts2(200, 14, -0.5, 0.5)
    Vt = torch.tensor(V, device="cuda", requires_grad=True)
    gt = torch.tensor(g, device="cuda", requires_grad=True)
    st = torch.tensor(src, device="cuda", requires_grad=True)
    scene = wos.Polyline(Vt, F, gt, source_type=2, source_params=st)
    fwd = wos.WoSWithSourceCUDA(nwalks=16, nsteps=64, use_IS_for_greens=True)
    bwd = wos.OursCUDA(nwalks=16, nsteps=64, epsilon=1e-3, epsilon2=1e-3, grad_values=True, grad_source=True,
                       use_IS_for_greens=True, source_in_normal_derivative=True)
    u = wos.CustomSolver(fwd, bwd).walk(P, scene, seed=9)
    (u * u).mean().backward()
    ns = scene._native
    s = fwd.walk_settings(scene, 9)
    mean = ns.solve(P, s)
    np.testing.assert_array_equal(_np(u), _np(mean.float()))
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=True)
    dV, dg, ds = ns.adjoint(P, s, a, (2.0 / len(P)) * mean.float())
    for x, y in ((Vt.grad, dV), (gt.grad, dg), (st.grad, ds)):
        np.testing.assert_allclose(_np(x), _np(y), rtol=1e-5, atol=1e-6 * np.abs(_np(y)).max())
    # the reference's default OursCUDA gives only the shape gradient
    Vt.grad = None
    gt.grad = None
    st.grad = None
    u2 = wos.CustomSolver(fwd, wos.OursCUDA(nwalks=16, nsteps=64, use_IS_for_greens=True)).walk(P, scene, seed=9)
    (u2 * u2).mean().backward()
    assert Vt.grad is not None and gt.grad is None and st.grad is None


def test_walk_detector_jittered_pixels(cuda, oracle):
    """Pixel sampling (wos/solver.py:67-84): each walk starts at a uniformly
    jittered point of its pixel; the image is the per-pixel mean, and its
    gradient runs the adjoint from the same jittered starts."""
    import torch
    import wos
    V, F, g = circle_scene(256)
    Vt = torch.tensor(V, device="cuda", requires_grad=True)
    scene = wos.Polyline(Vt, F, torch.tensor(g, device="cuda"))
    det = wos.Detector(vmin=(-0.8, -0.8), vmax=(0.8, 0.8), res=(24, 20))
    fwd = wos.WoSCUDA(nwalks=8, nsteps=64, epsilon=1e-3)
    bwd = wos.OursCUDA(nwalks=8, nsteps=64, epsilon=1e-3, epsilon2=1e-3)
    img = wos.CustomSolver(fwd, bwd).walk_detector(scene, det, seed=3)
    P = _np(det.make_points())
    s = fwd.walk_settings(scene, 3, jitter=det.jitter())
    assert s.jitter == (1.6 / 24, 1.6 / 20, 0.0)
    os_ = oracle.OracleScene(V, F, g)
    ov, _, _ = os_.walk_values(P, _oparams(oracle, s))
    om, _ = oracle.reduce(ov)
    np.testing.assert_allclose(_np(img), om.astype(np.float32), rtol=1e-6, atol=1e-7)
    # the jitter changes the walks: unjittered values differ
    assert not np.array_equal(_np(scene._native.solve(P, fwd.walk_settings(scene, 3))), om)
    (img * img).sum().backward()
    dLdu = (2.0 * om).astype(np.float32)
    a = bwd.adjoint_settings(scene, True, False, False)
    oa = oracle.make_adj(a.epsilon2, a.clamping, a.control_variates, a.source_in_normal_derivative, a.ball_epsilon,
                         True, False, False)
    odV, _, _ = os_.adjoint(P, _oparams(oracle, s), oa, dLdu)
    np.testing.assert_allclose(_np(Vt.grad), odV, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odV).max())
    assert wos.device_status() == 0


@pytest.mark.parametrize("kind", ["circle", "sphere"])
def test_projected_walk_adjoint_matches_oracle(cuda, oracle, kind):
    """Walks that reach nsteps are projected to their closest boundary point
    (the Dr.Jit WoS, wos/wos.py:43) in the primal walk and in the walks on the
    inscribed ball, as the reference's Ours does (wos/wos_grad.py:57-86);
    nsteps 6 makes many walks end that way."""
    from wos.native import AdjointSettings
    V, F, g = {"circle": lambda: circle_scene(256), "sphere": lambda: sphere_scene(2)}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(200, 13, -0.6, 0.6) if V.shape[1] == 2 else _pts3(150, 13, -0.5, 0.5)
    rng = np.random.default_rng(13)
    dLdu = rng.normal(size=len(P)).astype(np.float32)
    s = _settings(nwalks=8, nsteps=6, seed=17, project_unterminated=True)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True)
    dV, dg, _ = ns.adjoint(P, s, a, dLdu)
    odV, odg, _ = os_.adjoint(P, _oparams(oracle, s), oracle.make_adj(1e-3, 0.1, True, False, 1e-3, True, True, False),
                              dLdu)
    np.testing.assert_allclose(_np(dV), odV, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odV).max())
    np.testing.assert_allclose(_np(dg), odg, rtol=GRAD_RTOL, atol=GRAD_RTOL * np.abs(odg).max())
    # records at a single walk: the normal derivative with projected ball walks
    s1 = _settings(nwalks=1, nsteps=6, seed=18, project_unterminated=True)
    orec = os_.walk_records(P, _oparams(oracle, s1))
    nd = _np(ns.normal_derivative(orec, s1, a))
    assert np.array_equal(nd, os_.normal_derivative(orec, _oparams(oracle, s1), oracle.make_adj(1e-3, 0.1)))


@pytest.mark.parametrize("kind", ["circle", "sphere"])
def test_normal_derivative_given_radius_bit_exact(cuda, oracle, kind):
    """wos_normal_derivative_radius (override_R): with R the inscribed radius
    it is wos_normal_derivative; with other radii it equals the oracle's."""
    from wos.native import AdjointSettings
    V, F, g = {"circle": circle_scene, "sphere": sphere_scene}[kind]()
    ns, os_ = _scenes(oracle, V, F, g)
    P = _pts2(400, 19, -0.7, 0.7) if V.shape[1] == 2 else _pts3(300, 19, -0.6, 0.6)
    s = _settings(nwalks=1, nsteps=64, seed=23)
    orec = os_.walk_records(P, _oparams(oracle, s))
    a = AdjointSettings(epsilon2=5e-4, clamping=0.1)
    R = _np(ns.inscribed_ball(orec["valid"], orec["pt"], orec["n"]))
    assert np.array_equal(_np(ns.normal_derivative(orec, s, a, R=R)), _np(ns.normal_derivative(orec, s, a)))
    R2 = (0.5 * R).astype(np.float32)
    nd = _np(ns.normal_derivative(orec, s, a, R=R2))
    ond = os_.normal_derivative(orec, _oparams(oracle, s), oracle.make_adj(5e-4, 0.1), R=R2)
    assert np.array_equal(nd, ond)
