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
        """du/dn at boundary records (wos/wos.py:184-232): off-centred Poisson
        kernel on the largest inscribed ball, two antithetic samples, each a
        full walk at this solver's epsilon.  Returns (grad * n_x, grad * n_y)
        with n the outward normal."""
        if override_R is not None:
            raise NotImplementedError("override_R is not supported; the ball radius is always the inscribed one")
        s = as_sampler(sampler)
        st = self.walk_settings(scene, s.seed, nwalks=1, walk_offset=s.take())
        a = AdjointSettings(epsilon2=float(self.epsilon), clamping=float(clamping),
                            control_variates=bool(control_variates),
                            source_in_normal_derivative=bool(self.source_in_normal_derivative))
        out = scene._native.normal_derivative(its.as_dict(), st, a)
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


@dataclass
class Baseline(Solver):
    """Soft-edge fully differentiated walk (wos/wos.py:158-187) is a
    comparison estimator outside the hot path; not provided."""
    epsilon: float = 0.005
    nwalks: int = 10
    nsteps: int = 32

    def walk(self, p, scene, seed=0):
        raise NotImplementedError("Baseline is not part of the B200 hot path")
