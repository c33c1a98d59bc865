"""3D walk-on-spheres solvers (reference: wos/wos3d.py)."""
from __future__ import annotations

from dataclasses import dataclass

from .native import AdjointSettings
from .solver import Solver, as_sampler


@dataclass
class WoS3D(Solver):
    epsilon: float = 1e-3
    nwalks: int = 10
    nsteps: int = 32
    double_sided: bool = False

    project_unterminated = True

    def normal_derivative(self, its, scene, sampler, clamping=1e-1):
        """du/dn at boundary records (wos/wos3d.py:97-135): kernel
        P = -1 / (sqrt(2) (1 - cos theta)^1.5), cos theta clamped to
        1 - clamping, antithetic azimuth phi + pi.  Returns grad * n."""
        s = as_sampler(sampler)
        st = self.walk_settings(scene, s.seed, nwalks=1, walk_offset=s.take())
        a = AdjointSettings(epsilon2=float(self.epsilon), clamping=float(clamping), control_variates=True)
        out = scene._native.normal_derivative(its.as_dict(), st, a)
        return out[:, 0], out[:, 1], out[:, 2]

    def grad(self, p, scene, sampler):
        """One finite-shell estimate of grad u per point (wos/wos3d.py:66-95):
        two antithetic walks from the first ball with a control variate."""
        from .gradient import finite_shell_grad
        return finite_shell_grad(self, p, scene, sampler, with_source=False)

    def tangent_derivative(self, its, scene, sampler=None):
        return scene.tangent_derivative(its)


@dataclass
class WoS3DCUDA(WoS3D):
    prevent_fd_artifacts: bool = False

    project_unterminated = False
