"""The CPU oracle against the reference's golden data and known answers.

Pins: the reference's tabulated Green's-function CDF, the reference's
point-triangle routine (both generated by tests/golden/make_golden.py),
Philox-4x32-10 known-answer vectors (Random123), and analytic solutions of
the Laplace / Poisson problems the reference's ablations use
(ablations/test_disk.py:15-37, ablations/test_clover.py:16-46).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def test_g_cdf_matches_reference_table(oracle):
    ref = json.load(open(GOLD / "g_cdf_ref.json"))
    cdf = oracle.g_cdf(ref["size"])
    idx = np.array(ref["index"])
    # the reference prints 8 decimals; regenerated from its formula in double
    np.testing.assert_allclose(cdf[idx], np.array(ref["value"]), rtol=0, atol=5e-7)
    # non-decreasing; the last entries tie in float32 (pmf ~ r log(1/r) -> 0)
    assert cdf[-1] == 1.0 and np.all(np.diff(cdf) >= 0)


def test_point_triangle_matches_reference(oracle):
    z = np.load(GOLD / "ericson_ref.npz")
    uv, d = oracle.tri_closest(z["a"], z["b"], z["c"], z["p"])
    # same Voronoi-region algorithm, different float association
    np.testing.assert_allclose(uv, z["uv"], atol=1e-4, rtol=0)
    np.testing.assert_allclose(d, z["d"], atol=2e-6, rtol=1e-5)


@pytest.mark.parametrize("key,ctr,expect", [
    ((0, 0), (0, 0, 0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff), (0xffffffff,) * 4, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0xa4093822, 0x299f31d0), (0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(oracle, key, ctr, expect):
    # the library keys Philox with (seed_lo, seed_hi ^ 0x5bd1e995)
    seed = ((key[1] ^ 0x5bd1e995) << 32) | key[0]
    out = oracle.philox(seed, np.array([ctr], np.uint32))[0]
    assert tuple(int(v) for v in out) == expect


def _circle_oracle(oracle, n=1024, g_fn=None, source=None):
    from wos import shapes
    V, F = shapes.circle(n)
    g = g_fn(V) if g_fn is not None else shapes.harmonic_c1(V)
    if source is None:
        return oracle.OracleScene(V, F, g.astype(np.float32))
    return oracle.OracleScene(V, F, g.astype(np.float32), *source)


def test_oracle_harmonic_closed_form_c1(oracle):
    """Circle, g = x^3 - 3xy^2: the walk mean is unbiased (RMSE ~ SE)."""
    from wos import shapes
    S = _circle_oracle(oracle)
    P = shapes.grid(40, -0.9, 0.9)
    P = P[np.hypot(P[:, 0], P[:, 1]) < 1.0]
    vals, valid, steps = S.walk_values(P, oracle.make_params(nwalks=256, nsteps=256, epsilon=1e-3, seed=0))
    mean, var = oracle.reduce(vals)
    se = np.sqrt(var / 256)
    err = mean - shapes.harmonic_c1(P)
    # epsilon-shell bias is O(eps |grad u|) ~ 3e-3 next to the boundary
    assert np.all(np.abs(err) < 5.0 * se + 5e-3)
    assert np.sqrt((err ** 2).mean()) < 1.2 * np.sqrt((se ** 2).mean()) + 1e-3
    assert (steps == 256).mean() < 1e-3


def test_oracle_poisson_constant_source_disk(oracle):
    """Unit disk, g = 0, f = 1: u = (1 - r^2) / 4; uniform and G-importance-sampled source terms."""
    from wos import shapes
    S = _circle_oracle(oracle, g_fn=lambda V: np.zeros(len(V)), source=(2, [0, 0, 0, 0, 1.0]))
    P = np.array([[0.0, 0.0], [0.3, -0.2], [-0.5, 0.5], [0.7, 0.1]], np.float32)
    exact = (1 - (P ** 2).sum(1)) / 4
    for use_IS in (False, True):
        prm = oracle.make_params(nwalks=20000, nsteps=256, seed=1, include_source=True, use_IS_for_greens=use_IS)
        vals, _, _ = S.walk_values(P, prm)
        mean, var = oracle.reduce(vals)
        se = np.sqrt(var / 20000)
        assert np.all(np.abs(mean - exact) < 4.5 * se + 2e-3), (use_IS, mean, exact, se)


def test_oracle_fp64_reference_solution(oracle):
    """The FP64 reference solver (used where no closed form exists): unbiased
    on the circle for the harmonic x^3 - 3xy^2 (f = 0) and for u = (1 - r^2)/4
    (g = 0, f = 1, source term by its expectation R^2 / 4 per step)."""
    from wos import shapes
    P = np.array([[0.0, 0.0], [0.3, -0.2], [-0.5, 0.4], [0.7, 0.1], [0.1, 0.85]])
    S = _circle_oracle(oracle)
    mean, var, trunc = S.solve_f64(P, 8192, 0.0, seed=1)
    se = np.sqrt(var / 8192)
    assert trunc == 0
    assert np.all(np.abs(mean - shapes.harmonic_c1(P)) < 4.0 * se + 2e-3), (mean, se)
    S0 = _circle_oracle(oracle, g_fn=lambda V: np.zeros(len(V)))
    mean, var, trunc = S0.solve_f64(P, 8192, 1.0, seed=2)
    se = np.sqrt(var / 8192)
    exact = (1 - (P ** 2).sum(1)) / 4
    assert np.all(np.abs(mean - exact) < 4.0 * se + 1e-3), (mean, exact, se)


def test_oracle_poisson_sinusoid_source(oracle):
    """u = sin(3x + 4y) solves -Lap u = 25 sin(3x + 4y) (source type 2)."""
    from wos import shapes
    S = _circle_oracle(oracle, g_fn=lambda V: np.sin(3 * V[:, 0] + 4 * V[:, 1]),
                       source=(2, [3.0, 4.0, 0.0, 25.0, 0.0]))
    P = np.array([[0.1, 0.2], [-0.4, 0.3], [0.5, -0.5]], np.float32)
    prm = oracle.make_params(nwalks=20000, nsteps=256, seed=2, include_source=True, use_IS_for_greens=True)
    vals, _, _ = S.walk_values(P, prm)
    mean, var = oracle.reduce(vals)
    se = np.sqrt(var / 20000)
    exact = np.sin(3 * P[:, 0] + 4 * P[:, 1])
    assert np.all(np.abs(mean - exact) < 4.5 * se + 5e-3), (mean, exact, se)


def test_oracle_normal_derivative_disk(oracle):
    """u = r^4 cos(4 theta) on the unit disk: du/dn = 4 cos(4 theta)
    (ablations/test_disk.py:15-37)."""
    S = _circle_oracle(oracle, g_fn=lambda V: np.cos(4 * np.arctan2(V[:, 1], V[:, 0])))
    theta = np.array([0.3, 1.1, 2.5])
    P = np.stack([0.999 * np.cos(theta), 0.999 * np.sin(theta)], 1).astype(np.float32)
    c = S.closest(P)
    n = 4000
    rec = dict(valid=np.ones(len(P) * n, np.uint8), pt=np.repeat(c["pt"], n, 0), n=np.repeat(c["n"], n, 0),
               tuv=np.repeat(c["tuv"], n, 0), prim=np.repeat(c["prim"], n, 0))
    out = S.normal_derivative(rec, oracle.make_params(nsteps=256, seed=3), oracle.make_adj(1e-4, 1e-2))
    # grad * n_out dotted with the outward normal (-record normal)
    g = -(out * rec["n"]).sum(1).reshape(len(P), n)
    mean, se = g.mean(1), g.std(1) / np.sqrt(n)
    exact = 4 * np.cos(4 * theta)
    assert np.all(np.abs(mean - exact) < 5 * se + 0.05), (mean, exact, se)


@pytest.mark.parametrize("R", [0.25, 0.6])
def test_oracle_normal_derivative_given_radius_disk(oracle, R):
    """override_R (wos/wos.py:71-74): on any ball inside the domain tangent
    at the boundary point the estimator stays unbiased; the same disk problem
    as above on balls of radius R instead of the inscribed one."""
    S = _circle_oracle(oracle, g_fn=lambda V: np.cos(4 * np.arctan2(V[:, 1], V[:, 0])))
    theta = np.array([0.3, 1.1, 2.5])
    P = np.stack([0.999 * np.cos(theta), 0.999 * np.sin(theta)], 1).astype(np.float32)
    c = S.closest(P)
    n = 4000
    rec = dict(valid=np.ones(len(P) * n, np.uint8), pt=np.repeat(c["pt"], n, 0), n=np.repeat(c["n"], n, 0),
               tuv=np.repeat(c["tuv"], n, 0), prim=np.repeat(c["prim"], n, 0))
    out = S.normal_derivative(rec, oracle.make_params(nsteps=256, seed=5), oracle.make_adj(1e-4, 1e-2), R=R)
    g = -(out * rec["n"]).sum(1).reshape(len(P), n)
    mean, se = g.mean(1), g.std(1) / np.sqrt(n)
    exact = 4 * np.cos(4 * theta)
    assert np.all(np.abs(mean - exact) < 5 * se + 0.05), (mean, exact, se)


def test_oracle_harmonic_3d(oracle):
    """Displaced icosphere, g = x^2 - y^2 + z."""
    from wos import shapes
    V, F = shapes.displaced_icosphere(3, 0.15, 0)
    S = oracle.OracleScene(V, F, shapes.harmonic_c3(V).astype(np.float32))
    P = np.array([[0.0, 0.0, 0.0], [0.2, -0.3, 0.1], [-0.4, 0.2, 0.3]], np.float32)
    vals, _, _ = S.walk_values(P, oracle.make_params(nwalks=4000, nsteps=256, seed=4))
    mean, var = oracle.reduce(vals)
    se = np.sqrt(var / 4000)
    exact = shapes.harmonic_c3(P)
    assert np.all(np.abs(mean - exact) < 4.5 * se + 2e-3), (mean, exact, se)


def test_oracle_bvh_equals_brute(oracle):
    from wos import shapes
    V, F = shapes.star(2048)
    S = oracle.OracleScene(V, F, np.zeros(len(V), np.float32))
    rng = np.random.default_rng(0)
    P = rng.uniform(-1, 1, (5000, 2)).astype(np.float32)
    a, b = S.closest(P, use_bvh=True), S.closest(P, use_bvh=False)
    assert np.array_equal(a["prim"], b["prim"]) and np.array_equal(a["dist"], b["dist"])
    nb, npr = S.bvh_counts(P)
    assert nb.mean() < 100 and npr.mean() < 50  # logarithmic, not linear, work


def test_oracle_lbvh_structure(oracle):
    """Karras hierarchy: every leaf and internal node (except the root)
    appears exactly once as a child."""
    from wos import shapes
    V, F = shapes.displaced_icosphere(2, 0.15, 0)
    S = oracle.OracleScene(V, F, np.zeros(len(V), np.float32))
    ch, keys = S.bvh()
    n = len(F)
    assert ch.shape == (n - 1, 2)
    internal = ch[ch >= 0]
    leaves = ~ch[ch < 0]
    assert sorted(internal.tolist()) == list(range(1, n - 1))
    assert sorted(leaves.tolist()) == list(range(n))
    assert np.all(np.diff(keys.astype(np.uint64)) > 0)


def test_oracle_walk_from_a_nan_point_is_invalid(oracle):
    """A point with no primitive at a finite distance ends as an invalid walk
    (the kernels follow the same rule)."""
    import numpy as np
    from wos import shapes
    V, F = shapes.circle(64)
    S = oracle.OracleScene(V, F, np.ones(len(V), np.float32))
    P = np.array([[np.nan, 0.0], [0.0, 0.0]], np.float32)
    vals, valid, _ = S.walk_values(P, oracle.make_params(nwalks=2, nsteps=16, double_sided=True))
    assert not valid[0].any() and (vals[0] == 0).all()
    assert valid[1].all()
