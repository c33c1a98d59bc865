"""The CPU oracle against the reference's own estimators.

tests/golden/ref_estimators.npz holds per-point means and variances of the
reference's Python estimators, executed by tests/golden/make_golden.py on a
numpy stand-in for Dr.Jit (PCG32 random numbers):
  walk2 / walk3      WoS.single_walk (wos/wos.py:26-54), WoS3D.single_walk
                     (wos/wos3d.py:34-61)
  walk2_src[_is]     WoSWithSource.single_walk with a sinusoid source, uniform
                     and Green's-function importance sampling
                     (wos/wos_with_source.py:56-107)
  nd2 / nd2_src / nd3  normal_derivative at boundary records
                     (wos/wos.py:59-107, wos/wos_with_source.py:154-232,
                     wos/wos3d.py:97-135)
  ours2 / ours3      the boundary-shape estimator Ours.single_walk
                     (wos/wos_grad.py:57-86) and Ours3D.single_walk
                     (wos/wos_grad_3d.py:104-137), differentiated in forward
                     mode along a fixed vertex motion
  boundary2 / 3      WoSBoundary's derivative image (wos/wos_boundary.py:11-31)
                     for the same motion; 3D with the reference's pdf.
The oracle's Philox walks are a different random stream, so the comparison
is statistical: per-point means agree within their combined standard errors
(assert_same_expectation).  The same fixtures check the CUDA path in
tests/test_gpu_reference_estimators.py.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import assert_same_expectation

GOLD = Path(__file__).resolve().parent / "golden"
W2, W3 = 16384, 8192  # oracle walks per point


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(GOLD / "ref_estimators.npz"))


def _scene(oracle, ref, s, source=False):
    V, F, g = ref[s + "_V"], ref[s + "_F"], ref[s + "_g"]
    if source:
        return oracle.OracleScene(V, F, g, 2, ref["s2_source"])
    return oracle.OracleScene(V, F, g)


def _rec(ref, key, w):
    return {k: np.repeat(ref[f"{key}_{f}"], w, 0) for k, f in
            (("valid", "valid"), ("pt", "p"), ("n", "n"), ("tuv", "tuv"), ("prim", "prim"))}


def _se(ref, case, d):
    """Standard error of a fixture mean (per-walk variance / walks)."""
    return np.sqrt(ref[case + "_var"] / int(ref[f"s{d}_W"]))


def _mean_se(x):
    """Per-row mean and standard error of samples (rows x samples)."""
    x = np.asarray(x, np.float64)
    return x.mean(1), x.std(1, ddof=1) / np.sqrt(x.shape[1])


@pytest.mark.parametrize("case,src,IS", [("walk2", False, False), ("walk2_src", True, False),
                                         ("walk2_src_is", True, True)])
def test_oracle_walk_2d_matches_reference(oracle, ref, case, src, IS):
    S = _scene(oracle, ref, "s2", src)
    p = oracle.make_params(W2, 64, 1e-3, use_IS_for_greens=IS, include_source=src, project_unterminated=True, seed=1)
    vals, _, _ = S.walk_values(ref["s2_P"], p)
    m, se = _mean_se(vals)
    assert_same_expectation(m, se, ref[case + "_mean"], _se(ref, case, 2), case)


def test_oracle_walk_3d_matches_reference(oracle, ref):
    S = _scene(oracle, ref, "s3")
    vals, _, _ = S.walk_values(ref["s3_P"], oracle.make_params(W3, 128, 1e-3, project_unterminated=True, seed=2))
    m, se = _mean_se(vals)
    assert_same_expectation(m, se, ref["walk3_mean"], _se(ref, "walk3", 3), "walk3")


@pytest.mark.parametrize("case", ["nd2", "nd2_src", "nd3"])
def test_oracle_normal_derivative_matches_reference(oracle, ref, case):
    d3 = case == "nd3"
    src = case == "nd2_src"
    S = _scene(oracle, ref, "s3" if d3 else "s2", src)
    key = "rec3" if d3 else "rec2"
    n = len(ref[key + "_prim"])
    w = W3 if d3 else W2
    # the ball walks end like the reference's WoS walks: projected at nsteps
    p = oracle.make_params(1, 128 if d3 else 64, 1e-3, include_source=src, project_unterminated=True, seed=3)
    a = oracle.make_adj(1e-3, 0.1, True, src)
    nd = S.normal_derivative(_rec(ref, key, w), p, a).reshape(n, w, -1)
    m = nd.mean(1)
    se = nd.std(1, ddof=1) / np.sqrt(w)
    assert_same_expectation(m, se, ref[case + "_mean"], _se(ref, case, 3 if d3 else 2), case)


def test_oracle_inscribed_ball_matches_reference_radius(oracle, ref):
    """R of the reference's bisection (include/scene.cuh:225-249) at the same
    records; the reference value comes from the fixture generator's
    restatement over the reference's own Python sdf."""
    for d, key in ((2, "rec2"), (3, "rec3")):
        S = _scene(oracle, ref, f"s{d}")
        R = S.inscribed_ball(ref[key + "_valid"], ref[key + "_p"], ref[key + "_n"], 1e-3, use_bvh=True)
        np.testing.assert_allclose(R, ref[f"nd{d}_R"], rtol=2e-3)


@pytest.mark.parametrize("d", [2, 3])
def test_oracle_boundary_shape_estimator_matches_reference(oracle, ref, d):
    """Ours / Ours3D: the directional derivative of each point's mean along
    the vertex motion dV equals dV . (gradient of that mean), which the
    oracle's adjoint gives with dL/du = 1 at that point.  K independent
    batches of walks give the oracle's standard error."""
    S = _scene(oracle, ref, f"s{d}")
    P, dV = ref[f"s{d}_P"], ref[f"s{d}_dV"].astype(np.float64)
    K, w = 8, (W2 if d == 2 else W3) // 8
    a = oracle.make_adj(1e-3, 0.1, True, False, 1e-3, True, False, False)
    est = np.zeros((len(P), K))
    for i in range(len(P)):
        for k in range(K):
            p = oracle.make_params(w, 64 if d == 2 else 128, 1e-3, project_unterminated=True, walk_offset=k * w,
                                   seed=4)
            dVi, _, _ = S.adjoint(P[i:i + 1], p, a, np.ones(1, np.float32))
            est[i, k] = float((dVi * dV).sum())
    m, se = _mean_se(est)
    case = f"ours{d}"
    assert_same_expectation(m, se, ref[case + "_mean"], _se(ref, case, d), case)


@pytest.mark.parametrize("d", [2, 3])
def test_oracle_boundary_term_matches_reference(oracle, ref, d):
    """WoSBoundary's derivative image on an 8 x 8 detector over [-1, 1]^2
    (3D: Detector3D at z = 0.05, slab 0.25 thick, with the reference's pdf)."""
    S = _scene(oracle, ref, f"s{d}")
    if d == 2:
        det = oracle.make_detector(res=(8, 8))
    else:
        det = oracle.make_detector(res=(8, 8), slab_axis=2, slab_center=0.05, slab_half_width=0.125, flags=1)
    K, w = 8, 2048
    imgs = np.stack([S.boundary_term(det, w, seed=100 + k, dV_dir=ref[f"s{d}_dV"])[0] for k in range(K)], 1)
    m, se = _mean_se(imgs)
    case = f"boundary{d}"
    assert_same_expectation(m, se, ref[case + "_mean"], ref[case + "_se"], case)


def test_reference_3d_boundary_term_is_twice_the_area_pdf_term(oracle, ref):
    """The reference's Scene3D.sample_boundary divides the triangle pmf by
    |ab x ac| (wos/scene3d.py:251, :262), twice the area: its 3D boundary term
    is twice the one with the correct pdf 1 / (total area).  The comparison
    above has the power to tell the two apart."""
    S = _scene(oracle, ref, "s3")
    det = oracle.make_detector(res=(8, 8), slab_axis=2, slab_center=0.05, slab_half_width=0.125, flags=0)
    K, w = 8, 2048
    imgs = np.stack([S.boundary_term(det, w, seed=300 + k, dV_dir=ref["s3_dV"])[0] for k in range(K)], 1)
    m, se = _mean_se(imgs)
    assert_same_expectation(2 * m, 2 * se, ref["boundary3_mean"], ref["boundary3_se"], "2 x area-pdf term")
    with pytest.raises(AssertionError):
        assert_same_expectation(m, se, ref["boundary3_mean"], ref["boundary3_se"], "area-pdf term")
