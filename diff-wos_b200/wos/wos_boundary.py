"""Image-space boundary term of shape derivatives (wos/wos_boundary.py:11-31).

`WoSBoundary.walk_detector` returns a zero image attached to the scene's
vertex positions.  Its derivative is the boundary contribution to the pixel
integrals of u when the shape moves: boundary points are drawn uniformly by
length (2D) or area (3D), and each one that lands in a pixel adds
-g(x) (n . dx) / pdf / (detector size * nwalks) there.  Reverse mode (loss
.backward()) and forward mode (torch.autograd.forward_ad, the reference's
dr.forward_to renderings) both run wos_boundary_term.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .solver import Solver, has_tangent


class _BoundaryFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scene, detector, nwalks, seed, vertices, flags=0):
        ctx.scene, ctx.det, ctx.nwalks, ctx.seed, ctx.flags = scene, detector, nwalks, seed, flags
        ctx.vshape = vertices.shape
        npix = int(detector.res[0]) * int(detector.res[1])
        return torch.zeros(npix, dtype=torch.float32, device=vertices.device)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad):
        _, dV = ctx.scene._native.boundary_term(ctx.det.c(ctx.flags), ctx.nwalks, ctx.seed, dLdI=grad)
        return None, None, None, None, dV.reshape(ctx.vshape), None

    @staticmethod
    def jvp(ctx, _scene, _det, _nwalks, _seed, dV, _flags):
        if dV is None:
            return None
        img, _ = ctx.scene._native.boundary_term(ctx.det.c(ctx.flags), ctx.nwalks, ctx.seed, dV_dir=dV)
        return img.to(torch.float32)


@dataclass
class WoSBoundary(Solver):
    """The boundary term of the image derivative (diff_solve/runner.py:86-92
    adds it to the walk's derivative image).

    reference_area_pdf: in 3D, divide each sample's triangle pmf by
    |ab x ac| as the reference does (wos/scene3d.py:241-262).  That is twice
    the triangle's area, so the reference's 3D term is twice the correct
    one; the default uses the correct pdf 1 / (total area).  2D is the same
    either way (the reference divides by the segment length)."""
    reference_area_pdf: bool = False

    def flags(self) -> int:
        from ._lib import WOS_DETECTOR_REFERENCE_AREA_PDF
        return WOS_DETECTOR_REFERENCE_AREA_PDF if self.reference_area_pdf else 0

    def walk_detector(self, scene, detector, seed=0):
        V = scene.vertices
        if (torch.is_grad_enabled() and V.requires_grad) or has_tangent(V):
            return _BoundaryFunction.apply(scene, detector, int(self.nwalks), int(seed), V, self.flags())
        npix = int(detector.res[0]) * int(detector.res[1])
        return torch.zeros(npix, dtype=torch.float32, device=V.device)
