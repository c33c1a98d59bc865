"""The inverse problem on top of the fused forward + adjoint step: recover
per-vertex Dirichlet values from interior observations with Adam (the loop
of diff-wos inv_solve, seed = iteration).  The loss must fall by a large
factor and the recovered values must approach the truth."""
from __future__ import annotations

from pathlib import Path

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


def test_inverse_translation_converges(cuda):
    """A scene-transform inverse problem on top of the vertex adjoint
    (inv_solve/test_wrench.py:54-66): the boundary values ride with the
    vertices, so translating the shape by t moves the solution rigidly;
    Adam on t through torch autograd (CustomSolver with OursCUDA) recovers
    the target translation from interior observations."""
    import torch
    import wos
    from wos import shapes
    V0, F = shapes.star(1024, 0.6, 0.25, 5)
    g = (V0[:, 0] ** 2 - V0[:, 1] ** 2 + 0.5 * V0[:, 0] + 0.3 * V0[:, 1]).astype(np.float32)
    V0t = torch.tensor(V0, device="cuda")
    gt = torch.tensor(g, device="cuda")
    P = shapes.grid(40, -0.3, 0.3)
    Pd = torch.as_tensor(P, device="cuda")
    t_true = torch.tensor([0.05, -0.03], device="cuda")
    fwd = wos.WoSCUDA(nwalks=64, nsteps=64, epsilon=1e-3)
    target = fwd.solve(Pd, wos.Polyline(V0t + t_true, F, gt), seed=999)
    t = torch.zeros(2, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([t], lr=5e-3)
    sched = torch.optim.lr_scheduler.StepLR(opt, step_size=40, gamma=0.5)
    # The forward and the adjoint use the same walks (common random numbers,
    # the reference's CustomSolver), so the squared loss's gradient carries
    # the covariance of the two estimates, a bias of order 1/nwalks: 32 walks
    # settle about 0.013 from the target, 128 walks within the tolerance.
    solver = wos.CustomSolver(wos.WoSCUDA(nwalks=128, nsteps=64, epsilon=1e-3),
                              wos.OursCUDA(nwalks=128, nsteps=64, epsilon=1e-3, epsilon2=1e-3))
    tail = []
    for it in range(160):
        scene = wos.Polyline(V0t + t, F, gt)
        u = solver.walk(Pd, scene, seed=it)
        loss = ((u - target) ** 2).mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
        sched.step()
        if it >= 130:
            tail.append(t.detach().clone())
    t_avg = torch.stack(tail).mean(0)
    err = float(torch.linalg.norm(t_avg - t_true))
    assert err < 0.008, (t_avg.cpu().numpy(), err)
    assert wos.device_status() == 0


def _wrench_in_box(angle, shift):
    """inv_solve/test_wrench.py:54-66: the wrench (data/meshes/wrench.obj,
    flipped) rotated by `angle` and shifted, concatenated with the script's
    box polyline (its four corners as written there, the fourth repeating the
    second) scaled by 5, whose values are 0."""
    import torch
    from wos import io
    V, F, g = io.read_2d_obj(Path(__file__).resolve().parent / "golden" / "meshes" / "wrench.obj",
                             flip_orientation=True)
    V0 = torch.tensor(V, dtype=torch.float32, device="cuda")
    c, s = torch.cos(angle), torch.sin(angle)
    R = torch.stack([torch.stack([c, -s]), torch.stack([s, c])])
    shape = V0 @ R.T + shift
    box = torch.tensor([[-1.0, -1.0], [-1.0, 1.0], [1.0, 1.0], [-1.0, 1.0]], device="cuda") * 5.0
    verts = torch.cat([shape, box])
    faces = np.concatenate([F, np.array([[0, 1], [1, 2], [2, 3], [3, 0]]) + len(V)]).astype(np.int32)
    values = torch.cat([torch.tensor(g, dtype=torch.float32, device="cuda"), torch.zeros(4, device="cuda")])
    return verts, faces, values


def test_wrench_rotation_in_box_converges(cuda):
    """The reference's scene-transform inverse problem (inv_solve/test_wrench.py:
    12-115): observations on the boundary of [-1, 1]^2 (a 1024 grid's border,
    4,092 points), double-sided walks, L1 loss, Adam with lr 0.06 on the
    rotation and 1e-5 on the translation, the forward WoSCUDA with 100 walks
    and the gradient from OursCUDA with 10 walks, epsilon2 5e-4, clamping 0.1;
    the target rotation is pi / 2 from a start at 0."""
    import torch
    import wos
    x = np.linspace(-1.0, 1.0, 1024)
    X, Y = np.meshgrid(x, x)
    m = np.abs(np.maximum(np.abs(X), np.abs(Y)) - 1.0) < 1e-4
    Pd = torch.tensor(np.stack([X[m], Y[m]], 1), dtype=torch.float32, device="cuda")
    assert len(Pd) == 4092
    tgt = wos.Polyline(*_wrench_in_box(torch.tensor(np.pi / 2, device="cuda"), torch.zeros(2, device="cuda")))
    target = wos.WoSCUDA(nwalks=10000, nsteps=64, double_sided=True).solve(Pd, tgt, seed=12345)
    rot = torch.zeros((), device="cuda", requires_grad=True)
    shift = torch.zeros(2, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([rot], lr=0.06)
    opt2 = torch.optim.Adam([shift], lr=1e-5)
    solver = wos.CustomSolver(wos.WoSCUDA(nwalks=100, nsteps=64, double_sided=True),
                              wos.OursCUDA(nwalks=10, nsteps=64, double_sided=True, epsilon2=5e-4, clamping=0.1))
    losses, rots = [], []
    for it in range(200):
        scene = wos.Polyline(*_wrench_in_box(rot, shift))
        u = solver.walk(Pd, scene, seed=it)
        loss = (u - target).abs().sum()
        opt.zero_grad()
        opt2.zero_grad()
        loss.backward()
        opt.step()
        opt2.step()
        losses.append(float(loss))
        rots.append(float(rot))
    final = float(np.mean(rots[-20:]))
    assert abs(final - np.pi / 2) < 0.05, (final, rots[::20])
    assert np.mean(losses[-20:]) < 0.25 * losses[0], (losses[0], losses[-20:])
    assert wos.device_status() == 0
