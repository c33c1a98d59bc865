"""2D walk-on-spheres with an interior source term (reference:
wos/wos_with_source.py).

Each step adds f(y) G(y) / pdf(y) for one y in the step's ball, with y
uniform in the ball or, with use_IS_for_greens, radius drawn from the
tabulated CDF of r G(r) (include/wos.cuh:49-88 and :115-139).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .wos import WoS


@dataclass
class WoSWithSource(WoS):
    use_IS_for_greens: bool = False
    control_variates: bool = True
    source_epsilon: float = 0.0

    include_source = True
    differentiates_source = True  # the source term stays attached (wos/wos_with_source.py:89-90)
    source_in_normal_derivative = True

    def __post_init__(self):
        N = 10000
        r = (np.arange(N) + 0.5) / N
        pmf = r * np.log(1.0 / r) / (2.0 * np.pi)
        self.G_cdf = np.cumsum(pmf) / pmf.sum()
        self.step = 1.0 / N

    def grad(self, p, scene, sampler):
        """One finite-shell estimate of grad u per point
        (wos/wos_with_source.py:109-152): two antithetic walks from the
        first ball with a control variate, plus the interior source term."""
        from .gradient import finite_shell_grad
        return finite_shell_grad(self, p, scene, sampler, with_source=True)

    def eval_G(self, p, R, r_clamp=1e-4):
        """Green's function of the disk of radius R at distance |p| from its centre."""
        r = torch.linalg.norm(p, dim=-1)
        return torch.log(R / torch.clamp(r, min=r_clamp)) / (2.0 * np.pi)

    def eval_P(self, center, y, s, R):
        """Poisson kernel of the disk (wos/wos_with_source.py:38-45)."""
        y = y - center
        s = s - center
        r = torch.linalg.norm(y, dim=-1)
        c = (y * s).sum(-1) / torch.linalg.norm(s, dim=-1)
        denom = R * R - 2 * R * c + r * r
        return (R * R - r * r) / torch.clamp(denom, min=1e-5) / (2.0 * np.pi * R)


@dataclass
class WoSWithSourceCUDA(WoSWithSource):
    """The CUDA variant (wos/wos_with_source.py:235-265): its source term is
    detached, so only Dirichlet values receive gradients."""
    prevent_fd_artifacts: bool = False

    project_unterminated = False
    differentiates_source = False
