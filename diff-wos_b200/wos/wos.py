"""2D walk-on-spheres solvers (reference: wos/wos.py).

WoS and WoSCUDA run the same sm_100a kernel; they differ, as in the
reference, in what happens to a walk that reaches nsteps: the reference's
Dr.Jit WoS projects it to its closest boundary point (wos/wos.py:43), the CUDA
walk marks it invalid (include/wos.cuh:144).
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .native import AdjointSettings
from .solver import Solver, as_sampler


@dataclass
class WoS(Solver):
    epsilon: float = 1e-3
    nwalks: int = 10
    nsteps: int = 32
    double_sided: bool = False

    project_unterminated = True
    source_in_normal_derivative = False

    def normal_derivative(self, its, scene, sampler, override_R=None, clamping=1e-1, control_variates=True):
        """du/dn at boundary records (wos/wos.py:59-107): off-centred Poisson
        kernel on the largest inscribed ball (or on balls of radius override_R,
        a scalar or one per record), two antithetic samples, each a full walk
        at this solver's epsilon.  Returns (grad * n_x, grad * n_y) with n the
        outward normal."""
        s = as_sampler(sampler)
        st = self.walk_settings(scene, s.seed, nwalks=1, walk_offset=s.take())
        a = AdjointSettings(epsilon2=float(self.epsilon), clamping=float(clamping),
                            control_variates=bool(control_variates),
                            source_in_normal_derivative=bool(self.source_in_normal_derivative))
        out = scene._native.normal_derivative(its.as_dict(), st, a, R=override_R)
        return tuple(out[:, k] for k in range(scene.dim))

    def tangent_derivative(self, its, scene, sampler=None):
        return scene.tangent_derivative(its)

    def grad(self, p, scene, sampler):
        """One finite-shell estimate of grad u per point (the estimator of
        wos/wos_with_source.py:109-152 without its source term)."""
        from .gradient import finite_shell_grad
        return finite_shell_grad(self, p, scene, sampler, with_source=False)


@dataclass
class WoSCUDA(WoS):
    """WoS with the CUDA walk's semantics (wos/wos.py:136-155)."""
    prevent_fd_artifacts: bool = False

    project_unterminated = False


class _SoftFunction(torch.autograd.Function):
    """Per-point means of the soft-edge walk, differentiable in both modes:
    forward mode (the reference's renderD use of Baseline,
    diff_solve/runner.py:75-109) by wos_soft_walk's tangents, reverse mode by
    wos_soft_walk_adjoint (the reference's walk is a fully attached Dr.Jit
    computation, wos/wos.py:170-187)."""

    @staticmethod
    def forward(ctx, solver, scene, P, s, vertices, values):
        ctx.solver, ctx.scene, ctx.P, ctx.s = solver, scene, P, s
        return scene._native.soft_walk(P, s)["mean"].to(torch.float32)

    @staticmethod
    def jvp(ctx, _solver, _scene, _P, _s, dV, dg):
        out = ctx.scene._native.soft_walk(ctx.P, ctx.s, dV=dV, dg=dg, want_tangent=True)
        return out["tangent"].to(torch.float32)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad):
        need_V, need_g = ctx.needs_input_grad[4], ctx.needs_input_grad[5]
        dV, dg = ctx.scene._native.soft_walk_adjoint(ctx.P, ctx.s, grad, want_dV=need_V, want_dg=need_g)
        return None, None, None, None, dV, dg


class _SoftWalk:
    """The soft-edge walk (wos/wos.py:158-187, wos/wos_grad_3d.py:24-57):
    every walk takes nsteps steps, adding beta (1 - w) g with
    w = min(d, epsilon) / epsilon and then beta *= w.  Values and their
    forward-mode derivatives come from the wos_soft_walk kernel."""

    def soft_settings(self, scene, seed, jitter=None):
        from .native import WalkSettings
        return WalkSettings(nwalks=int(self.nwalks), nsteps=int(self.nsteps), epsilon=float(self.epsilon),
                            double_sided=bool(self.double_sided), use_bvh=bool(scene.use_bvh), seed=int(seed),
                            jitter=tuple(jitter) if jitter is not None else (0.0, 0.0, 0.0))

    def walk(self, p, scene, seed=0, jitter=None):
        from .fwd import points
        from .solver import has_tangent
        P = points(p, scene.dim)
        s = self.soft_settings(scene, seed, jitter)
        V, g = scene.vertices, scene.values
        if has_tangent(V) or has_tangent(g) or (torch.is_grad_enabled() and (V.requires_grad or g.requires_grad)):
            return _SoftFunction.apply(self, scene, P, s, V, g)
        return scene._native.soft_walk(P, s)["mean"].to(torch.float32)

    def solve(self, p, scene, seed=0, jitter=None):
        from .fwd import points
        return scene._native.soft_walk(points(p, scene.dim), self.soft_settings(scene, seed, jitter))["mean"].to(
            torch.float32)

    def walk_detector(self, scene, detector, seed=0):
        return self.walk(detector.make_points(), scene, seed, jitter=detector.jitter())


@dataclass
class Baseline(_SoftWalk, Solver):
    """Soft-edge walk on polylines (wos/wos.py:158-187)."""
    epsilon: float = 0.005
    nwalks: int = 10
    nsteps: int = 32
