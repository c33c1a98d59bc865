"""Finite-shell boundary-shape estimators the paper compares against
(Baseline2 / Baseline2CUDA, wos/wos_grad.py:14-112; Baseline23D,
wos/wos_grad_3d.py:60-100).

Each sample walks once from the query point to its boundary record (the GPU
walk kernel), nudges that boundary point by l into the domain, estimates
grad u there with the finite-shell estimator (two walks from the first
ball, wos/gradient.py), and contributes -(grad u) . dx to the gradient, with
dx the motion of the boundary point through the vertices (get_point).  The
value is zero; torch autograd carries the vertex gradient.  With
normal_derivative_only, grad u keeps its normal component from the
estimator and takes the tangential one from the boundary data.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .fwd import points
from .solver import Sampler, Solver, as_sampler


class _ShellBaseline(Solver):
    l: float = 5e-3
    normal_derivative_only: bool = False

    def _inner(self):
        raise NotImplementedError

    def single_walk(self, p, scene, sampler):
        s = as_sampler(sampler)
        P = points(p, scene.dim)
        inner = self._inner()
        with torch.no_grad():
            inside = torch.ones(P.shape[0], dtype=torch.bool, device=P.device)
            if not self.double_sided:
                inside = scene.is_inside(P)
            its = inner.single_walk_preliminary(P, scene, s)
        its_a = scene.get_point(its)
        with torch.no_grad():
            n = its.n
            p_in = its.p.detach() + n * float(self.l)
            g = torch.stack(inner.grad(p_in, scene, s), 1)
            if self.normal_derivative_only:
                gn = (g * n).sum(1, keepdim=True) * n
                gt = torch.stack(scene.tangent_derivative(its), 1)
                g = gn + gt
        v = its_a.p - its_a.p.detach()
        res = -(g * v).sum(1)
        ok = inside & its.valid
        return torch.where(ok, res, torch.zeros_like(res))

    def walk(self, p, scene, seed=0):
        """Mean over nwalks samples (zero value, vertex gradient attached)."""
        s = Sampler(seed)
        acc = None
        for _ in range(int(self.nwalks)):
            r = self.single_walk(p, scene, s)
            acc = r if acc is None else acc + r
        return acc / float(self.nwalks)

    def solve(self, p, scene, seed=0):
        return torch.zeros(points(p, scene.dim).shape[0], dtype=torch.float32, device=scene.vertices.device)


@dataclass
class Baseline2CUDA(_ShellBaseline):
    """2D finite-shell baseline on the CUDA walk (wos/wos_grad.py:14-50, 90-112)."""
    epsilon: float = 1e-3
    nwalks: int = 10
    nsteps: int = 32
    l: float = 5e-3
    normal_derivative_only: bool = False

    def _inner(self):
        from .wos_with_source import WoSWithSourceCUDA
        return WoSWithSourceCUDA(nwalks=1, nsteps=self.nsteps, epsilon=self.epsilon, double_sided=self.double_sided)


@dataclass
class Baseline2(Baseline2CUDA):
    """The reference's Dr.Jit Baseline2 runs the same estimator."""


@dataclass
class Baseline23D(_ShellBaseline):
    """3D finite-shell baseline (wos/wos_grad_3d.py:60-100)."""
    epsilon: float = 1e-3
    nwalks: int = 10
    nsteps: int = 32
    l: float = 5e-3
    normal_derivative_only: bool = False

    def _inner(self):
        from .wos3d import WoS3DCUDA
        return WoS3DCUDA(nwalks=1, nsteps=self.nsteps, epsilon=self.epsilon, double_sided=self.double_sided)
