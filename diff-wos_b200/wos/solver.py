"""Solver base class, the counter-based sampler and the autograd bridge
(reference: wos/solver.py, wos/fwd.py:44-105).

`walk(p, scene, seed)` returns per-point means over nwalks walks as a torch
float32 tensor.  When scene tensors (vertices, values, source_params) require
grad, the result is attached to them through one torch.autograd.Function
whose backward runs the adjoint kernel with the same seed -- the reference's
_CustomSolver.backward (wos/solver.py:109-114).  Walks are defined by their
Philox counters (common random numbers): the backward either repeats the
primal walks or, when forward and backward walk the same way, starts from the
boundary records the forward kept (8-16 bytes per walk); both give the same
gradients.
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum

import torch

from .fwd import points
from .native import AdjointSettings, WalkSettings


class ControlVarianceType(Enum):
    NoControlVariate = 0
    RunningControlVariate = 1
    BoundaryControlVariate = 2
    BoundaryAndRunningControlVariate = 3


class Sampler:
    """Counter-based stand-in for the reference's per-lane PCG32 sampler.

    A walk's random numbers are Philox(seed; point index, walk index, step,
    role); `offset` is the walk index the next single_walk call uses.  Like
    the reference's sampler, it advances in place on every call."""

    def __init__(self, seed: int = 0, offset: int = 0):
        self.seed = int(seed)
        self.offset = int(offset)

    def take(self, n: int = 1) -> int:
        o = self.offset
        self.offset += n
        return o


def as_sampler(sampler) -> Sampler:
    if isinstance(sampler, Sampler):
        return sampler
    return Sampler(int(sampler) if sampler is not None else 0)


@dataclass
class Solver:
    """Base solver (wos/solver.py:16-88).  Subclasses set the walk semantics
    through walk_settings() and, for differentiation, adjoint_settings()."""
    epsilon: float = 0.005  # shell width that stops a walk
    nwalks: int = 20  # walks per query point
    nsteps: int = 4  # maximum walk length
    double_sided: bool = False
    control_variance: ControlVarianceType = ControlVarianceType.NoControlVariate
    antithetic: bool = False

    # walk semantics of this solver family
    project_unterminated = True
    include_source = False
    differentiates_source = False

    def walk_settings(self, scene, seed=0, nwalks=None, walk_offset=0, jitter=None) -> WalkSettings:
        return WalkSettings(nwalks=int(self.nwalks if nwalks is None else nwalks), nsteps=int(self.nsteps),
                            epsilon=float(self.epsilon), double_sided=bool(self.double_sided),
                            prevent_fd_artifacts=bool(getattr(self, "prevent_fd_artifacts", False)),
                            use_IS_for_greens=bool(getattr(self, "use_IS_for_greens", False)),
                            include_source=bool(self.include_source and scene.source_type != 0),
                            project_unterminated=bool(self.project_unterminated), use_bvh=bool(scene.use_bvh),
                            walk_offset=int(walk_offset), seed=int(seed),
                            jitter=tuple(jitter) if jitter is not None else (0.0, 0.0, 0.0))

    def adjoint_settings(self, scene, want_dV, want_dg, want_dsrc) -> AdjointSettings:
        """Gradients this solver provides as a backward solver: the attached
        Dirichlet gather (values) and, for the source-differentiating solver,
        the source term."""
        return AdjointSettings(want_dV=False, want_dg=bool(want_dg),
                               want_dsrc=bool(want_dsrc and self.differentiates_source))

    # ------------------------------------------------------------ primal
    def solve(self, p, scene, seed=0, jitter=None) -> torch.Tensor:
        """Per-point means, detached (wos/solver.py:41-44).  `jitter`: per-axis
        extent of a uniform start-point offset per walk (pixel sampling)."""
        P = points(p, scene.dim)
        return scene._native.solve(P, self.walk_settings(scene, seed, jitter=jitter)).to(torch.float32)

    def solve_stats(self, p, scene, seed=0):
        """(mean, variance of the per-walk values), both float64."""
        P = points(p, scene.dim)
        return scene._native.solve(P, self.walk_settings(scene, seed), want_var=True)

    def walk(self, p, scene, seed=0, jitter=None) -> torch.Tensor:
        """Per-point means, attached to the scene's differentiable tensors
        (wos/solver.py:46-65)."""
        return _attach(self, self, p, scene, seed, jitter)

    def walk_reduce(self, p, scene, seed=0):
        return self.walk(p, scene, seed)

    def walk_detector(self, scene, detector, seed=0):
        """Per-pixel means over nwalks walks, each starting at a uniformly
        jittered point of its pixel (wos/solver.py:67-84)."""
        return self.walk(detector.make_points(), scene, seed, jitter=detector.jitter())

    def single_walk_preliminary(self, p, scene, sampler):
        """One walk per point; the boundary record (WoS.single_walk in
        wos_ext, include/wos.cuh:374-533)."""
        s = as_sampler(sampler)
        P = points(p, scene.dim)
        st = self.walk_settings(scene, s.seed, nwalks=1, walk_offset=s.take())
        o = scene._native.records(P, st)
        return _record(scene, o)

    def single_walk(self, p, scene, sampler):
        """One walk per point; its value (wos/wos.py:171-179)."""
        its = self.single_walk_preliminary(p, scene, sampler)
        val = scene.dirichlet(its)
        if self.include_source and scene.source_type != 0:
            val = val + torch.where(its.valid, its.contrib, torch.zeros_like(its.contrib))
        return val

    def u(self, p, scene, sampler):
        return self.single_walk(p, scene, sampler)

    def per_walk_values(self, p, scene, seed=0, with_steps=False):
        """(n, nwalks) per-walk values (0 for invalid walks)."""
        P = points(p, scene.dim)
        return scene._native.values(P, self.walk_settings(scene, seed), want_steps=with_steps)


def _record(scene, o):
    from .scene import ClosestPointRecord
    from .scene3d import ClosestPointRecord3D
    valid = o["valid"].bool()
    if scene.dim == 2:
        return ClosestPointRecord(valid=valid, p=o["pt"], n=o["n"], t=o["tuv"][:, 0].contiguous(),
                                  prim_id=o["prim"], contrib=o["contrib"])
    return ClosestPointRecord3D(valid=valid, p=o["pt"], n=o["n"], uv=o["tuv"], prim_id=o["prim"],
                                contrib=o["contrib"])


class _Job:
    """One differentiable walk: forward values from `fwd`, gradients from
    `bwd` with the same seed.  When both solvers walk with identical settings
    the forward keeps every walk's boundary record and the backward starts
    from it instead of repeating the primal walk (same result)."""

    def __init__(self, fwd, bwd, p, scene, seed, needs=(True, True, True), jitter=None):
        self.fwd, self.bwd, self.scene, self.seed = fwd, bwd, scene, seed
        self.P = points(p, scene.dim)
        self.records = None
        self.needs = needs
        self.jitter = jitter

    def forward(self):
        if self.fwd is None:
            return torch.zeros(self.P.shape[0], dtype=torch.float32, device=self.P.device)
        sf = self.fwd.walk_settings(self.scene, self.seed, jitter=self.jitter)
        sb = self.bwd.walk_settings(self.scene, self.seed, jitter=self.jitter)
        if sf == sb:
            a = self.bwd.adjoint_settings(self.scene, *self.needs)
            want_dc = bool(a.want_dsrc and sb.include_source and self.scene.source_type != 0 and self.scene.dim == 2)
            mean, _, rec, dc = self.scene._native.solve_records(self.P, sf, want_dcontrib=want_dc)
            self.records = (rec, dc)
            return mean.to(torch.float32)
        return self.fwd.solve(self.P, self.scene, self.seed, jitter=self.jitter)

    def tangent(self, dV, dg, ds):
        """Forward mode: derivative of the per-point means along (dV, dg, ds)
        (any may be None), from the backward solver's estimator with the same
        seed (wos_solve_tangent)."""
        s = self.bwd.walk_settings(self.scene, self.seed, jitter=self.jitter)
        a = self.bwd.adjoint_settings(self.scene, dV is not None, dg is not None, ds is not None)
        if not (a.want_dV or a.want_dg or a.want_dsrc):
            return torch.zeros(self.P.shape[0], dtype=torch.float32, device=self.P.device)
        out = self.scene._native.solve_tangent(self.P, s, a, dV=dV if a.want_dV else None,
                                               dg=dg if a.want_dg else None, dsrc=ds if a.want_dsrc else None)
        return out["tangent"].to(torch.float32)

    def backward(self, grad, need_V, need_g, need_s):
        s = self.bwd.walk_settings(self.scene, self.seed, jitter=self.jitter)
        a = self.bwd.adjoint_settings(self.scene, need_V, need_g, need_s)
        if not (a.want_dV or a.want_dg or a.want_dsrc):
            return None, None, None
        g = grad.to(torch.float32).contiguous()
        if self.records is not None and (self.records[1] is not None or not a.want_dsrc or
                                         not (s.include_source and self.scene.source_type != 0)):
            dV, dg, ds = self.scene._native.adjoint_records(self.P, s, a, g, *self.records)
        else:
            dV, dg, ds = self.scene._native.adjoint(self.P, s, a, g)
        self.records = None
        if ds is not None and self.scene.source_params is None:
            ds = None
        return dV, dg, ds


class _WalkFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, job, vertices, values, source_params):
        ctx.job = job
        ctx.shapes = (vertices.shape, values.shape, source_params.shape)
        return job.forward()

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad):
        nV, ng, ns = ctx.needs_input_grad[1:]
        dV, dg, ds = ctx.job.backward(grad, nV, ng, ns)
        dV = dV.reshape(ctx.shapes[0]) if (nV and dV is not None) else None
        dg = dg.reshape(ctx.shapes[1]) if (ng and dg is not None) else None
        ds = ds.reshape(ctx.shapes[2]) if (ns and ds is not None) else None
        return None, dV, dg, ds

    @staticmethod
    def jvp(ctx, _job, dV, dg, ds):
        return ctx.job.tangent(dV, dg, ds)


def has_tangent(t) -> bool:
    """True for a forward-mode dual tensor (torch.autograd.forward_ad)."""
    return isinstance(t, torch.Tensor) and torch.autograd.forward_ad.unpack_dual(t).tangent is not None


def _attach(fwd, bwd, p, scene, seed, jitter=None):
    tensors = (scene.vertices, scene.values, scene.source_params_tensor())
    if any(has_tangent(t) for t in tensors) or (torch.is_grad_enabled() and any(t.requires_grad for t in tensors)):
        needs = tuple(bool(t.requires_grad) or has_tangent(t) for t in tensors)
        return _WalkFunction.apply(_Job(fwd, bwd, p, scene, seed, needs, jitter), *tensors)
    if fwd is None:
        return torch.zeros(points(p, scene.dim).shape[0], dtype=torch.float32, device=scene.vertices.device)
    return fwd.solve(p, scene, seed, jitter=jitter)


@dataclass
class CustomSolver:
    """Forward values from fwd_solver, gradients from bwd_solver with the same
    seed (wos/solver.py:90-125)."""
    fwd_solver: Solver = None
    bwd_solver: Solver = None

    def walk(self, p, scene, seed=0, jitter=None):
        return _attach(self.fwd_solver, self.bwd_solver, p, scene, seed, jitter)

    def walk_detector(self, scene, detector, seed=0):
        return self.walk(detector.make_points(), scene, seed, jitter=detector.jitter())

    def solve(self, p, scene, seed=0):
        return self.fwd_solver.solve(p, scene, seed)
