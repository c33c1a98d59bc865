"""Accuracy of the library's own elementary functions (wos_math.h), measured
against the C library in double precision.  The same source runs in the
kernels; these are the functions the walk samples directions, Green's
function values and source terms with."""
from __future__ import annotations

import numpy as np


def test_sincos_2pi(oracle):
    u = np.concatenate([np.linspace(0, 1, 200001), np.arange(0, 1 << 23, 997) / float(1 << 23)]).astype(np.float32)
    sc = oracle.math_fn("sincos_2pi", u)
    ang = 2 * np.pi * u.astype(np.float64)
    assert np.abs(sc[:, 0] - np.sin(ang)).max() < 3e-7
    assert np.abs(sc[:, 1] - np.cos(ang)).max() < 3e-7
    # exact symmetry points
    e = oracle.math_fn("sincos_2pi", np.array([0.0, 0.25, 0.5, 0.75, 1.0], np.float32))
    assert e[0, 0] == 0 and e[0, 1] == 1 and e[1, 1] == 0 and e[2, 0] == 0 and e[3, 1] == 0


def test_sin_cos_general(oracle):
    x = np.linspace(-60, 60, 400001).astype(np.float32)
    xd = x.astype(np.float64)
    assert np.abs(oracle.math_fn("sin", x) - np.sin(xd)).max() < 4e-7
    assert np.abs(oracle.math_fn("cos", x) - np.cos(xd)).max() < 4e-7


def test_log(oracle):
    x = np.concatenate([np.geomspace(1e-38, 1e38, 300001), np.linspace(0.5, 2, 100001),
                        [1.0, 2.0, 1e-40, 1e-44]]).astype(np.float32)
    r = oracle.math_fn("log", x)
    ref = np.log(x.astype(np.float64))
    assert np.all(np.abs(r - ref) <= 2.5e-7 * np.maximum(np.abs(ref), 1.0))
    assert r[np.where(x == 1.0)[0][0]] == 0.0


def test_exp(oracle):
    x = np.linspace(-87, 88, 400001).astype(np.float32)
    r = oracle.math_fn("exp", x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    assert np.all(np.abs(r - ref) <= 3e-7 * ref)
    assert oracle.math_fn("exp", np.array([0.0], np.float32))[0] == 1.0


def test_atan2(oracle):
    rng = np.random.default_rng(0)
    y = rng.normal(size=200000).astype(np.float32)
    x = rng.normal(size=200000).astype(np.float32)
    r = oracle.math_fn("atan2", y, x)
    assert np.abs(r - np.arctan2(y.astype(np.float64), x.astype(np.float64))).max() < 5e-7
