"""The inverse problem on top of the fused forward + adjoint step: recover
per-vertex Dirichlet values from interior observations with Adam (the loop
of diff-wos inv_solve, seed = iteration).  The loss must fall by a large
factor and the recovered values must approach the truth."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_inverse_values_converge(cuda):
    import torch
    import wos
    from wos import shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    V, F = shapes.star(1024, 0.6, 0.25, 5)
    th = np.arctan2(V[:, 1], V[:, 0])
    g_true = (np.cos(2 * th) + 0.5 * np.sin(3 * th)).astype(np.float32)
    P = shapes.grid(96, -1.0, 1.0)
    P = np.ascontiguousarray(P[shapes.inside_star(P, 0.6, 0.25, 5)])
    Pd = torch.as_tensor(P, device="cuda")
    target = NativeScene(V, F, g_true).solve(Pd, WalkSettings(nwalks=512, nsteps=64, seed=99)).float()
    scene = NativeScene(V, F, np.zeros_like(g_true))
    g = torch.zeros(len(g_true), device="cuda", requires_grad=True)
    opt = torch.optim.Adam([g], lr=5e-2)
    adj = AdjointSettings(want_dV=False, want_dg=True, want_dsrc=False)
    losses = []
    for it in range(150):
        out = scene.solve_adjoint(Pd, WalkSettings(nwalks=32, nsteps=64, seed=it), adj, loss_kind=2, target=target)
        losses.append(float(out["loss"]))
        opt.zero_grad(set_to_none=False)
        g.grad = out["dg"]
        opt.step()
        with torch.no_grad():
            scene.update_values(g.detach())
    gt = torch.as_tensor(g_true, device="cuda")
    err = float(torch.linalg.norm(g.detach() - gt) / torch.linalg.norm(gt))
    assert np.mean(losses[-10:]) < 0.15 * losses[0], (losses[0], losses[-10:])
    assert err < 0.6, err
    assert wos.device_status() == 0
