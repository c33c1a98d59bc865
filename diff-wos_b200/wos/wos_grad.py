"""Gradient solvers (reference: wos/wos_grad.py).

OursCUDA is the paper's boundary-shape estimator: a detached primal walk to
the boundary, the boundary point re-attached to the vertices (get_point), and
a Monte Carlo estimate of grad u there (normal derivative on the inscribed
ball + tangential derivative of the data); its walk() value is zero with the
shape gradient attached (wos/wos_grad.py:113-151).  Here the whole estimator
is one adjoint kernel launch per backward pass.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .native import AdjointSettings
from .solver import Solver, _attach


@dataclass
class OursCUDA(Solver):
    epsilon2: float = 1e-3
    clamping: float = 1e-1
    control_variates: bool = True
    # extensions beyond the reference, all defaulting to its behaviour: also
    # return the Dirichlet-value and source-parameter gradients of the primal
    # walk, and use the source-aware normal derivative
    # (wos/wos_with_source.py:154-232) when the scene has a source.  The
    # reference's OursCUDA calls WoSCUDA.normal_derivative, which ignores f
    # (wos/wos_grad.py:126, :146), so its shape gradient is biased when
    # f != 0; source_in_normal_derivative=True removes that bias.
    grad_values: bool = False
    grad_source: bool = False
    source_in_normal_derivative: bool = False
    use_IS_for_greens: bool = False

    project_unterminated = False
    include_source = True
    differentiates_source = True

    def adjoint_settings(self, scene, want_dV, want_dg, want_dsrc) -> AdjointSettings:
        return AdjointSettings(epsilon2=float(self.epsilon2), clamping=float(self.clamping),
                               control_variates=bool(self.control_variates),
                               source_in_normal_derivative=bool(self.source_in_normal_derivative),
                               want_dV=bool(want_dV), want_dg=bool(want_dg and self.grad_values),
                               want_dsrc=bool(want_dsrc and self.grad_source))

    def walk(self, p, scene, seed=0, jitter=None):
        """Zero-valued per-point result carrying the gradient."""
        return _attach(None, self, p, scene, seed, jitter)

    def solve(self, p, scene, seed=0, jitter=None):
        from .fwd import points
        return torch.zeros(points(p, scene.dim).shape[0], dtype=torch.float32, device=scene.vertices.device)


@dataclass
class Ours(OursCUDA):
    """The reference's pure-Dr.Jit Ours (wos/wos_grad.py:57-86): the same
    boundary-shape estimator on WoS walks, so the primal walk and the two
    walks on the inscribed ball all stop at this solver's epsilon (there is
    no epsilon2) and a walk that reaches nsteps is projected to its closest
    boundary point (wos/wos.py:43) instead of being dropped; the normal
    derivative is WoS.normal_derivative (wos/wos.py:59-107), which has no
    source term."""
    source_in_normal_derivative: bool = False

    project_unterminated = True

    def adjoint_settings(self, scene, want_dV, want_dg, want_dsrc) -> AdjointSettings:
        a = super().adjoint_settings(scene, want_dV, want_dg, want_dsrc)
        a.epsilon2 = float(self.epsilon)
        return a
