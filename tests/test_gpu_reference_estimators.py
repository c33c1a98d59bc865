"""The CUDA path against the reference's own estimators.

The fixtures (tests/golden/ref_estimators.npz) are per-point means and
variances of the reference's Python estimators, executed by
tests/golden/make_golden.py on a numpy stand-in for Dr.Jit; the cases are
listed in tests/test_reference_estimators.py, which checks the CPU oracle
against the same numbers.  Here every estimate comes from the C ABI
(libwos_b200.so) with the settings of the reference class that made the
fixture: WoS walks stop at epsilon and are projected to their closest
boundary point at nsteps (wos/wos.py:43, wos/wos3d.py:50), the normal
derivative uses the same epsilon and clamping 0.1, and the boundary-shape
estimator is the reference's Ours (wos/wos_grad.py:57-86: WoS walks at
epsilon for the primal and the ball walks).  Random streams differ (Philox
here, PCG32 there), so means are compared within their combined standard
errors (assert_same_expectation); the tangential derivative and the
inscribed-ball radius are deterministic and compared directly.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import assert_same_expectation

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
WG = 65536  # walks per point on the GPU


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(GOLD / "ref_estimators.npz"))


def _np(t):
    return t.detach().cpu().numpy()


def _native(ref, d, source=False):
    from wos.native import NativeScene
    s = f"s{d}"
    if source:
        return NativeScene(ref[s + "_V"], ref[s + "_F"], ref[s + "_g"], 2, ref["s2_source"])
    return NativeScene(ref[s + "_V"], ref[s + "_F"], ref[s + "_g"])


def _ref_se(ref, case, d):
    return np.sqrt(ref[case + "_var"] / int(ref[f"s{d}_W"]))


def _settings(**kw):
    from wos.native import WalkSettings
    kw.setdefault("epsilon", 1e-3)
    kw.setdefault("project_unterminated", True)
    return WalkSettings(**kw)


@pytest.mark.parametrize("case,d,src,IS", [("walk2", 2, False, False), ("walk2_src", 2, True, False),
                                           ("walk2_src_is", 2, True, True), ("walk3", 3, False, False)])
def test_walk_matches_reference(cuda, ref, case, d, src, IS):
    ns = _native(ref, d, src)
    s = _settings(nwalks=WG, nsteps=64 if d == 2 else 128, use_IS_for_greens=IS, include_source=src, seed=101)
    mean, var = ns.solve(ref[f"s{d}_P"], s, want_var=True)
    assert_same_expectation(_np(mean), np.sqrt(_np(var) / WG), ref[case + "_mean"], _ref_se(ref, case, d), case)


@pytest.mark.parametrize("case", ["nd2", "nd2_src", "nd3"])
def test_normal_derivative_matches_reference(cuda, ref, case):
    from wos.native import AdjointSettings
    d = 3 if case == "nd3" else 2
    src = case == "nd2_src"
    ns = _native(ref, d, src)
    key = f"rec{d}"
    n = len(ref[key + "_prim"])
    rec = {k: np.repeat(ref[f"{key}_{f}"], WG // 4, 0) for k, f in
           (("valid", "valid"), ("pt", "p"), ("n", "n"), ("tuv", "tuv"), ("prim", "prim"))}
    s = _settings(nwalks=1, nsteps=64 if d == 2 else 128, include_source=src, seed=102)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, control_variates=True, source_in_normal_derivative=src)
    nd = _np(ns.normal_derivative(rec, s, a)).astype(np.float64).reshape(n, WG // 4, d)
    m, se = nd.mean(1), nd.std(1, ddof=1) / np.sqrt(WG // 4)
    assert_same_expectation(m, se, ref[case + "_mean"], _ref_se(ref, case, d), case)


def test_inscribed_ball_and_tangent_derivative_match_reference(cuda, ref):
    """R at the fixture's records (include/scene.cuh:225-249, bisection
    resolution ~1e-3 of the extent) and the tangential derivative of the data
    (wos/scene.py:451-460, wos/wos3d.py:137-156), computed by the reference's
    own code in the fixture."""
    import torch
    import wos
    for d in (2, 3):
        ns = _native(ref, d)
        key = f"rec{d}"
        R = _np(ns.inscribed_ball(ref[key + "_valid"], ref[key + "_p"], ref[key + "_n"], 1e-3))
        np.testing.assert_allclose(R, ref[f"nd{d}_R"], rtol=2e-3)
        dev = dict(device="cuda")
        if d == 2:
            scene = wos.Polyline(torch.tensor(ref["s2_V"], **dev), torch.tensor(ref["s2_F"], **dev),
                                 torch.tensor(ref["s2_g"], **dev))
            its = wos.ClosestPointRecord(valid=torch.tensor(ref[key + "_valid"], **dev).bool(),
                                         p=torch.tensor(ref[key + "_p"], **dev), n=torch.tensor(ref[key + "_n"], **dev),
                                         t=torch.tensor(ref[key + "_tuv"][:, 0], **dev),
                                         prim_id=torch.tensor(ref[key + "_prim"], **dev))
            got = np.stack([_np(x) for x in scene.tangent_derivative(its)], 1)
            np.testing.assert_allclose(got, ref["tangent2"], rtol=1e-5, atol=1e-6)
        else:
            scene = wos.Scene3D(torch.tensor(ref["s3_V"], **dev), torch.tensor(ref["s3_F"], **dev),
                                torch.tensor(ref["s3_g"], **dev))
            its = wos.ClosestPointRecord3D(valid=torch.tensor(ref[key + "_valid"], **dev).bool(),
                                           p=torch.tensor(ref[key + "_p"], **dev),
                                           n=torch.tensor(ref[key + "_n"], **dev),
                                           uv=torch.tensor(ref[key + "_tuv"], **dev),
                                           prim_id=torch.tensor(ref[key + "_prim"], **dev))
            got = np.stack([_np(x) for x in wos.WoS3D().tangent_derivative(its, scene)], 1)
            np.testing.assert_allclose(got, ref["tangent3"], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("d", [2, 3])
def test_boundary_shape_estimator_matches_reference(cuda, ref, d):
    """The per-point directional derivative along the fixture's vertex motion
    (wos_solve_tangent), with the reference Ours' walks: projected WoS walks at
    epsilon for the primal and the ball walks."""
    import torch
    from wos.native import AdjointSettings
    ns = _native(ref, d)
    s = _settings(nwalks=WG, nsteps=64 if d == 2 else 128, seed=103)
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, control_variates=True, source_in_normal_derivative=False,
                        want_dV=True, want_dg=False)
    t = ns.solve_tangent(ref[f"s{d}_P"], s, a, dV=torch.tensor(ref[f"s{d}_dV"], device="cuda"), want_var=True)
    case = f"ours{d}"
    assert_same_expectation(_np(t["tangent"]), np.sqrt(_np(t["tangent_var"]) / WG), ref[case + "_mean"],
                            _ref_se(ref, case, d), case)


@pytest.mark.parametrize("d", [2, 3])
def test_boundary_term_matches_reference(cuda, ref, d):
    """WoSBoundary's derivative image (8 x 8 pixels over [-1, 1]^2; 3D:
    Detector3D at z = 0.05 with the reference's |ab x ac| pdf)."""
    import torch
    import wos
    ns = _native(ref, d)
    if d == 2:
        det = wos.Detector(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(8, 8))
    else:
        det = wos.Detector3D(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(8, 8), z=0.05)
    c = det.c(wos.WoSBoundary(reference_area_pdf=True).flags())
    dV = torch.tensor(ref[f"s{d}_dV"], device="cuda")
    K = 8
    imgs = np.stack([_np(ns.boundary_term(c, 16384, 200 + k, dV_dir=dV)[0]) for k in range(K)], 1)
    m, se = imgs.mean(1), imgs.std(1, ddof=1) / np.sqrt(K)
    case = f"boundary{d}"
    assert_same_expectation(m, se, ref[case + "_mean"], ref[case + "_se"], case)
    assert wos.device_status() == 0
