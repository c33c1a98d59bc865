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
