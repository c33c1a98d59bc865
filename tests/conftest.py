"""Test configuration: import paths, markers and shared fixtures.

`-m gpu` tests need a CUDA device and the built libwos_b200.so; everything
else runs on the CPU (oracle against golden vectors, host logic, C-ABI
symbol checks).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "diff-wos_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwos_b200.so")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import wos
    wos._lib.lib()
    wos.device_status(reset=True)
    return torch


def circle_scene(n=1024):
    from wos import shapes
    V, F = shapes.circle(n)
    g = shapes.harmonic_c1(V).astype(np.float32)
    return V, F, g


def star_scene(n=4096):
    from wos import shapes
    V, F = shapes.star(n)
    g = (np.sin(3 * V[:, 0]) * np.cos(2 * V[:, 1])).astype(np.float32)
    return V, F, g


def sphere_scene(subdiv=3, amplitude=0.15, seed=0):
    from wos import shapes
    V, F = shapes.displaced_icosphere(subdiv, amplitude, seed)
    g = shapes.harmonic_c3(V).astype(np.float32)
    return V, F, g


def assert_same_expectation(a, se_a, b, se_b, what="", z_max=4.5):
    """Two Monte Carlo estimates of the same per-point expectations agree:
    with z = (a - b) / sqrt(se_a^2 + se_b^2) per entry, at most
    max(1, 3 %) of the entries have |z| >= 3, none has |z| >= z_max, and
    mean(z^2) stays below the 99.99 % quantile of chi^2_n / n (a shared bias
    of about one standard error fails that).  Entries that both estimates
    give exactly (zero standard errors) must be equal."""
    from scipy.stats import chi2
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    s = np.hypot(np.asarray(se_a, np.float64).ravel(), np.asarray(se_b, np.float64).ravel())
    exact = s == 0
    assert np.all(a[exact] == b[exact]), f"{what}: deterministic entries differ"
    z = (a[~exact] - b[~exact]) / s[~exact]
    n = z.size
    assert n > 0
    msg = f"{what}: n={n} max|z|={np.abs(z).max():.2f} mean z^2={np.mean(z * z):.2f} z={np.round(z, 2)}"
    assert np.count_nonzero(np.abs(z) >= 3) <= max(1, int(0.03 * n)), msg
    assert np.abs(z).max() < z_max, msg
    assert np.mean(z * z) < chi2.ppf(0.9999, n) / n, msg
