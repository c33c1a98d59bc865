"""3D gradient solver (reference: wos/wos_grad_3d.py:104-137)."""
from __future__ import annotations

from dataclasses import dataclass

from .solver import Solver
from .wos import _SoftWalk
from .wos_grad import OursCUDA


@dataclass
class Ours3D(OursCUDA):
    """Boundary-shape estimator on triangle meshes: the 3D normal derivative
    (wos/wos3d.py:97-135) plus the face tangential derivative
    (wos/wos3d.py:137-156)."""
    epsilon2: float = 1e-3
    clamping: float = 1e-1


@dataclass
class Baseline3D(_SoftWalk, Solver):
    """Soft-edge walk on triangle meshes (wos/wos_grad_3d.py:24-57)."""
    epsilon: float = 0.005
    nwalks: int = 10
    nsteps: int = 32
