"""Finite-shell estimator of the spatial gradient of u at interior points
(WoSWithSource.grad, wos/wos_with_source.py:109-152; WoS3D.grad,
wos/wos3d.py:66-95; Monte Carlo geometry processing, eq. 13).

With R the distance from x to the boundary and w a uniform direction,
grad u(x) ~ (dim / R) w (u(x + R w) - u_ref), averaged with the antithetic
direction -w; u_ref = g at the closest boundary point (control variate).
In 2D a source adds the interior term f(y) pi R^2 grad G(x, y) with y uniform
in the ball.  Points within epsilon of the boundary (or outside, unless the
solver is double-sided) get 0.  The walks from the ball points run on the
GPU kernel with the solver's settings; the directions come from a CUDA
generator seeded by (seed, sampler offset).
"""
from __future__ import annotations

import math

import torch

from .fwd import points
from .solver import as_sampler


def finite_shell_grad(solver, p, scene, sampler, with_source: bool):
    s = as_sampler(sampler)
    dim = scene.dim
    P = points(p, dim)
    n = P.shape[0]
    dev = P.device
    off = s.take()
    rec = scene._native.closest(P, scene.use_bvh, want=("sdf", "inside"))
    R = rec["sdf"].abs()
    active = R >= float(solver.epsilon)
    if not solver.double_sided:
        active &= rec["inside"].bool()
    uref = scene.dirichlet(scene.closest_point(P)).detach()
    gen = torch.Generator(device=dev)
    gen.manual_seed((int(s.seed) * 0x9E3779B1 + off * 0x85EBCA77 + 0x27D4EB2F) & 0x7FFFFFFFFFFFFFFF)
    if dim == 2:
        th = 2.0 * math.pi * torch.rand(n, generator=gen, device=dev)
        w = torch.stack([torch.cos(th), torch.sin(th)], 1)
    else:
        z = 1.0 - 2.0 * torch.rand(n, generator=gen, device=dev)
        ph = 2.0 * math.pi * torch.rand(n, generator=gen, device=dev)
        rr = torch.sqrt(torch.clamp(1.0 - z * z, min=0.0))
        w = torch.stack([rr * torch.cos(ph), rr * torch.sin(ph), z], 1)
    Rc = R.unsqueeze(1)
    Y = torch.cat([P + Rc * w, P - Rc * w]).contiguous()
    st = solver.walk_settings(scene, s.seed, nwalks=1, walk_offset=off)
    uY = scene._native.values(Y, st)[:, 0]
    u_plus, u_minus = uY[:n] - uref, uY[n:] - uref
    G = (dim / R).unsqueeze(1) * w
    g = 0.5 * (G * u_plus.unsqueeze(1) - G * u_minus.unsqueeze(1))
    if with_source and dim == 2 and scene.source_type != 0:
        rho = torch.sqrt(torch.rand(n, generator=gen, device=dev))
        ph = 2.0 * math.pi * torch.rand(n, generator=gen, device=dev)
        y = P + Rc * rho.unsqueeze(1) * torch.stack([torch.cos(ph), torch.sin(ph)], 1)
        d = y - P
        r2 = (d * d).sum(1).clamp_min(1e-12)
        grad_G = d / (2.0 * math.pi) * (1.0 / r2 - 1.0 / (R * R)).unsqueeze(1)
        f = scene.source_function(y).detach()
        g = g + (f * math.pi * R * R).unsqueeze(1) * grad_G
    g = torch.where(active.unsqueeze(1), g, torch.zeros_like(g))
    return tuple(g[:, k] for k in range(dim))
