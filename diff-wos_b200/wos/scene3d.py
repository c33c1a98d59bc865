"""3D triangle-mesh scenes (reference: wos/scene3d.py)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .fwd import points, tensor
from .native import NativeScene
from .scene import Detector


@dataclass
class Detector3D(Detector):
    """Slab detector at height z (wos/scene3d.py:9-46)."""
    res: tuple = (256, 256)
    z: float = 0.05

    def __post_init__(self):
        self.l_z = (self.vmax[0] - self.vmin[0]) / self.res[0]

    def size(self):
        return float(np.prod(np.subtract(self.vmax, self.vmin))) * self.l_z

    def make_points(self) -> torch.Tensor:
        p = super().make_points()
        z = torch.full((p.shape[0], 1), float(self.z), device=p.device)
        return torch.cat([p, z], 1).contiguous()

    def c(self, flags: int = 0):
        """Slab |z - self.z| < l_z / 2 (wos/scene3d.py:35-41)."""
        d = super().c(flags)
        d.slab_axis, d.slab_center, d.slab_half_width = 2, float(self.z), float(self.l_z) / 2
        return d


@dataclass
class Detector3DY(Detector):
    """Slab detector at y = const (wos/scene3d.py:48-85)."""
    res: tuple = (256, 256)
    y: float = 0.05

    def __post_init__(self):
        self.l_y = (self.vmax[0] - self.vmin[0]) / self.res[0]

    def make_points(self) -> torch.Tensor:
        p = super().make_points()
        y = torch.full((p.shape[0],), float(self.y), device=p.device)
        return torch.stack([p[:, 0], y, p[:, 1]], 1).contiguous()

    def jitter(self):
        """x and z jitter (wos/scene3d.py:65-71)."""
        dx, dz = self.pixel()
        return (dx, 0.0, dz)

    def size(self):
        """Slab volume (image area x l_y)."""
        return float(np.prod(np.subtract(self.vmax, self.vmin))) * self.l_y

    def c(self, flags: int = 0):
        """Image axes x, z; slab |y - self.y| < l_y / 2 (wos/scene3d.py:73-81)."""
        d = super().c(flags)
        d.axis_u, d.axis_v = 0, 2
        d.slab_axis, d.slab_center, d.slab_half_width = 1, float(self.y), float(self.l_y) / 2
        return d


@dataclass
class ClosestPointRecord3D:
    """Boundary record (wos/scene3d.py:87-103); uv = (w_b, w_c)."""
    valid: torch.Tensor = None
    p: torch.Tensor = None
    n: torch.Tensor = None
    uv: torch.Tensor = None
    val: torch.Tensor = None
    prim_id: torch.Tensor = None
    J: torch.Tensor = None
    contrib: torch.Tensor = None

    def as_dict(self):
        return dict(valid=self.valid.to(torch.uint8), pt=self.p, n=self.n, tuv=self.uv, prim=self.prim_id)


class Scene3D:
    """Triangle-mesh boundary with per-vertex Dirichlet values
    (wos/scene3d.py:106-274; native side include/scene.cuh:316-495).
    vertices (nV, 3), indices (nF, 3) outward-oriented, values (nV,)."""

    dim = 3

    def __init__(self, vertices, indices, values, use_bvh=True):
        self.vertices = tensor(vertices, torch.float32).reshape(-1, 3)
        self.indices = tensor(indices, torch.int32).reshape(-1, 3).contiguous()
        self.values = tensor(values, torch.float32).reshape(-1)
        self.source_type = 0
        self.source_params = None
        self.use_bvh = bool(use_bvh)
        self._native = NativeScene(self.vertices.detach(), self.indices, self.values.detach())
        self.normals = self._native.normals()
        info = self._native.info()
        self.aabb = (torch.tensor(list(info.aabb_min)), torch.tensor(list(info.aabb_max)))
        self.bvh_nodes = int(info.n_nodes)
        self.bvh_depth = int(info.bvh_depth)
        self.init_dist()

    @staticmethod
    def from_obj(filename, normalize=True, flip_orientation=False, **kw):
        """OBJ triangle mesh (`v`, `f`, `c` lines), optionally centred and
        scaled to unit radius in double precision.  The reference's
        Scene3D.from_obj keeps only two coordinates per vertex
        (wos/scene3d.py:127) and cannot build a 3D scene; this reads all three,
        as its read_3d_obj does (wos/io.py:54-71).  A file without `c` lines
        gets zero values."""
        from .io import normalize_vertices, read_3d_obj
        V, F, g = read_3d_obj(filename, flip_orientation=flip_orientation)
        V = normalize_vertices(V) if normalize else V.astype(np.float32)
        g = g.astype(np.float32) if len(g) == len(V) else np.zeros(len(V), np.float32)
        return Scene3D(V, F.astype(np.int32), g, **kw)

    def update_values(self, values):
        self.values = tensor(values, torch.float32).reshape(-1)
        self._native.update_values(self.values.detach())

    def update_vertices(self, vertices):
        self.vertices = tensor(vertices, torch.float32).reshape(-1, 3)
        self._native.update_vertices(self.vertices.detach())
        self.normals = self._native.normals()
        info = self._native.info()
        self.aabb = (torch.tensor(list(info.aabb_min)), torch.tensor(list(info.aabb_max)))
        self.init_dist()

    def source_params_tensor(self) -> torch.Tensor:
        return torch.zeros(0, device=self.vertices.device)

    def init_dist(self):
        f = self.indices.long()
        V = self.vertices.detach()
        self.areas = torch.linalg.norm(torch.cross(V[f[:, 1]] - V[f[:, 0]], V[f[:, 2]] - V[f[:, 0]], dim=1), dim=1)

    def closest_point_preliminary(self, p) -> torch.Tensor:
        return self._native.closest(points(p, 3), self.use_bvh, want=("prim",))["prim"]

    def closest_point(self, p, active=None) -> ClosestPointRecord3D:
        o = self._native.closest(points(p, 3), self.use_bvh, want=("prim", "tuv", "pt", "n"))
        valid = o["prim"] >= 0
        if active is not None:
            valid = valid & active
        its = ClosestPointRecord3D(valid=valid, p=o["pt"], n=o["n"], uv=o["tuv"], prim_id=o["prim"])
        its.val = self.dirichlet(its)
        return its

    def sdf(self, p, active=None) -> torch.Tensor:
        return self._native.sdf(points(p, 3), self.use_bvh)

    def is_inside(self, p) -> torch.Tensor:
        return self._native.closest(points(p, 3), self.use_bvh, want=("inside",))["inside"].bool()

    def largest_inscribed_ball(self, its: ClosestPointRecord3D, epsilon=1e-3) -> torch.Tensor:
        return self._native.inscribed_ball(its.valid.to(torch.uint8), its.p.detach(), its.n.detach(), epsilon,
                                           self.use_bvh)

    def dirichlet(self, its: ClosestPointRecord3D) -> torch.Tensor:
        """b u + c v + a (1 - u - v) (wos/scene3d.py:216-223); attached to values."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        va, vb, vc = self.values[f[:, 0]], self.values[f[:, 1]], self.values[f[:, 2]]
        u, v = its.uv[:, 0], its.uv[:, 1]
        val = vb * u + vc * v + va * (1 - u - v)
        return torch.where(its.valid, val, torch.zeros_like(val))

    def get_point(self, its: ClosestPointRecord3D) -> ClosestPointRecord3D:
        """p = interpolate(a, b, c, uv) with uv detached (wos/scene3d.py:225-239)."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        uv = its.uv.detach()
        a, b, c = self.vertices[f[:, 0]], self.vertices[f[:, 1]], self.vertices[f[:, 2]]
        u, v = uv[:, :1], uv[:, 1:]
        p = b * u + c * v + a * (1 - u - v)
        va, vb, vc = self.values[f[:, 0]], self.values[f[:, 1]], self.values[f[:, 2]]
        val = vb * u[:, 0] + vc * v[:, 0] + va * (1 - u[:, 0] - v[:, 0])
        return ClosestPointRecord3D(valid=its.valid, p=p, n=its.n, uv=uv, val=val, prim_id=its.prim_id)

    def tangent_derivative(self, its: ClosestPointRecord3D):
        """Tangential gradient from the face's value slope (wos/wos3d.py:137-156)."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        V = self.vertices.detach()
        g = self.values.detach()
        a, b, c = V[f[:, 0]], V[f[:, 1]], V[f[:, 2]]
        ab, ac = b - a, c - a
        t = ab / torch.linalg.norm(ab, dim=1, keepdim=True)
        fn = torch.cross(ab, ac, dim=1)
        fn = fn / torch.linalg.norm(fn, dim=1, keepdim=True)
        n = torch.cross(fn, t, dim=1)
        n = n / torch.linalg.norm(n, dim=1, keepdim=True)
        gt = (g[f[:, 1]] - g[f[:, 0]]) / torch.linalg.norm(ab, dim=1)
        gn = ((g[f[:, 2]] - g[f[:, 0]]) - gt * (ac * t).sum(1)) / (ac * n).sum(1)
        out = gt[:, None] * t + gn[:, None] * n
        return out[:, 0], out[:, 1], out[:, 2]

    def write_obj(self, filename):
        from .io import write_3d_obj
        write_3d_obj(filename, self.vertices.detach().cpu().numpy(), self.indices.cpu().numpy(),
                     self.values.detach().cpu().numpy())
