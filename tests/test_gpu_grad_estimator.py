"""The finite-shell gradient estimator (WoSWithSource.grad, WoS3D.grad)
against closed forms: harmonic u = x^2 - y^2 on the unit disk, the Poisson
problem u = (1 - r^2) / 4 (f = 1) on the unit disk, and u = x^2 - y^2 + z on
the unit sphere; the mean over samples must match within a few standard
errors."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mean_se(solver, P, scene, nsamp):
    import torch
    from wos import Sampler
    s = Sampler(seed=11)
    acc = []
    for _ in range(nsamp):
        g = solver.grad(P, scene, s)
        acc.append(torch.stack(g, 1).cpu().numpy())
    a = np.stack(acc)
    return a.mean(0), a.std(0) / np.sqrt(nsamp)


@pytest.mark.parametrize("case", ["harmonic", "poisson"])
def test_grad_2d_closed_form(cuda, case):
    import torch
    import wos
    from wos import shapes
    V, F = shapes.circle(1024)
    if case == "harmonic":
        g = V[:, 0] ** 2 - V[:, 1] ** 2
        scene = wos.Polyline(torch.tensor(V), F, torch.tensor(g.astype(np.float32)))
    else:
        g = np.zeros(len(V), np.float32)
        scene = wos.Polyline(torch.tensor(V), F, torch.tensor(g), source_type=2,
                             source_params=torch.tensor([0.0, 0.0, 0.0, 0.0, 1.0]))
    rng = np.random.default_rng(3)
    P = rng.uniform(-0.5, 0.5, (64, 2)).astype(np.float32)
    solver = wos.WoSWithSourceCUDA(nwalks=1, nsteps=128, epsilon=1e-3)
    m, se = _mean_se(solver, P, scene, 400)
    exact = np.stack([2 * P[:, 0], -2 * P[:, 1]], 1) if case == "harmonic" else -0.5 * P
    z = (m - exact) / np.maximum(se, 1e-6)
    assert np.sqrt((z ** 2).mean()) < 1.6, np.sqrt((z ** 2).mean())
    assert np.abs(m - exact).max() < 6 * se.max() + 0.02


def test_grad_3d_closed_form(cuda):
    import torch
    import wos
    from wos import shapes
    V, F = shapes.icosphere(4)
    g = (V[:, 0] ** 2 - V[:, 1] ** 2 + V[:, 2]).astype(np.float32)
    scene = wos.Scene3D(torch.tensor(V), F, torch.tensor(g))
    rng = np.random.default_rng(4)
    P = rng.uniform(-0.4, 0.4, (48, 3)).astype(np.float32)
    solver = wos.WoS3DCUDA(nwalks=1, nsteps=128, epsilon=1e-3)
    m, se = _mean_se(solver, P, scene, 400)
    exact = np.stack([2 * P[:, 0], -2 * P[:, 1], np.ones(len(P))], 1)
    z = (m - exact) / np.maximum(se, 1e-6)
    assert np.sqrt((z ** 2).mean()) < 1.6, np.sqrt((z ** 2).mean())


def test_grad_zero_in_shell_and_outside(cuda):
    import torch
    import wos
    from wos import shapes
    V, F = shapes.circle(256)
    scene = wos.Polyline(torch.tensor(V), F, torch.tensor(np.ones(len(V), np.float32)))
    P = np.array([[0.0, 0.9995], [1.5, 0.0], [0.0, 0.0]], np.float32)
    gx, gy = wos.WoSWithSourceCUDA(nwalks=1, nsteps=256, epsilon=1e-3).grad(P, scene, 0)
    assert float(gx[0]) == 0.0 and float(gy[0]) == 0.0   # within epsilon of the boundary
    assert float(gx[1]) == 0.0 and float(gy[1]) == 0.0   # outside
    # constant boundary data: u = 1, grad = 0 (the control variate cancels exactly)
    assert abs(float(gx[2])) < 1e-5 and abs(float(gy[2])) < 1e-5
