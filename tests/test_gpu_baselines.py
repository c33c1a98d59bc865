"""The finite-shell baselines (Baseline2CUDA, Baseline23D) estimate the same
shape derivative as OursCUDA: for a translated shape whose values ride with
its vertices, d/dt of mean(u) over interior points is -mean(grad u . e).
u = x^2 - y^2 on the unit circle (2D) and x^2 - y^2 + z on the unit sphere
(3D), translation e = x: the exact derivative is -2 mean(x) (2D) and
-2 mean(x) (3D)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _translation_derivative(solver, make_scene, P, seed=1):
    import torch
    V, scene = make_scene()
    out = solver.walk(P, scene, seed=seed)
    assert float(out.detach().abs().max()) == 0.0
    out.mean().backward()
    return float(V.grad[:, 0].sum())


def test_baseline2_translation_derivative(cuda):
    import torch
    import wos
    from wos import shapes
    Vn, F = shapes.circle(1024)
    g = (Vn[:, 0] ** 2 - Vn[:, 1] ** 2).astype(np.float32)

    def make_scene():
        V = torch.tensor(Vn, device="cuda", requires_grad=True)
        return V, wos.Polyline(V, F, torch.tensor(g, device="cuda"))

    rng = np.random.default_rng(8)
    P = np.stack([rng.uniform(0.1, 0.5, 256), rng.uniform(-0.3, 0.3, 256)], 1).astype(np.float32)
    exact = -2.0 * P[:, 0].mean()
    est = [_translation_derivative(wos.Baseline2CUDA(nwalks=50, nsteps=128), make_scene, P, seed=s)
           for s in range(4)]
    ours = _translation_derivative(wos.CustomSolver(None, wos.OursCUDA(nwalks=200, nsteps=128)), make_scene, P)
    m, se = np.mean(est), np.std(est) / np.sqrt(len(est))
    assert abs(m - exact) < 4 * se + 0.05, (est, exact)
    assert abs(ours - exact) < 0.05, (ours, exact)


def test_baseline23d_translation_derivative(cuda):
    import torch
    import wos
    from wos import shapes
    Vn, F = shapes.icosphere(4)
    g = (Vn[:, 0] ** 2 - Vn[:, 1] ** 2 + Vn[:, 2]).astype(np.float32)

    def make_scene():
        V = torch.tensor(Vn, device="cuda", requires_grad=True)
        return V, wos.Scene3D(V, F, torch.tensor(g, device="cuda"))

    rng = np.random.default_rng(9)
    P = np.stack([rng.uniform(0.1, 0.4, 128), rng.uniform(-0.3, 0.3, 128), rng.uniform(-0.3, 0.3, 128)],
                 1).astype(np.float32)
    exact = -2.0 * P[:, 0].mean()
    est = [_translation_derivative(wos.Baseline23D(nwalks=50, nsteps=128), make_scene, P, seed=s) for s in range(4)]
    m, se = np.mean(est), np.std(est) / np.sqrt(len(est))
    assert abs(m - exact) < 4 * se + 0.06, (est, exact)
