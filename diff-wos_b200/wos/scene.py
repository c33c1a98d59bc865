"""2D scenes: Detector, closest-point records and Polyline
(reference: wos/scene.py).

Polyline keeps the reference's fields (vertices, indices, values, normals,
aabb, use_bvh, source_type, source_params) as torch CUDA tensors; queries run
in libwos_b200.so.  Tensors passed in with requires_grad=True stay attached:
solvers differentiate through them (values, source_params, vertices).
"""
from __future__ import annotations

import ctypes

from dataclasses import dataclass, field

import numpy as np
import torch

from .fwd import points, tensor
from .native import NativeScene


@dataclass
class Detector:
    """Pixel grid on [vmin, vmax] (wos/scene.py:9-42)."""
    vmin: tuple = (-1.0, -1.0)
    vmax: tuple = (1.0, 1.0)
    res: tuple = (100, 100)

    def size(self):
        return float(np.prod(np.subtract(self.vmax, self.vmin)))

    def pixel(self):
        """Pixel extent per image axis."""
        return tuple(float(b - a) / r for a, b, r in zip(self.vmin, self.vmax, self.res))

    def jitter(self):
        """Start-point jitter of pixel sampling (wos/scene.py:33-39)."""
        dx, dy = self.pixel()
        return (dx, dy, 0.0)

    def c(self, flags: int = 0):
        """The detector for the C ABI (wos_detector); flags: WOS_DETECTOR_* bits."""
        from ._lib import WosDetector
        return WosDetector((ctypes.c_float * 2)(*self.vmin), (ctypes.c_float * 2)(*self.vmax),
                           (ctypes.c_int32 * 2)(*self.res), 0, 1, -1, 0.0, 0.0, float(self.size()), int(flags))

    def make_points(self) -> torch.Tensor:
        x = torch.linspace(self.vmin[0], self.vmax[0], self.res[0], device="cuda")
        y = torch.linspace(self.vmax[1], self.vmin[1], self.res[1], device="cuda")  # flip y
        Y, X = torch.meshgrid(y, x, indexing="ij")
        return torch.stack([X.reshape(-1), Y.reshape(-1)], 1).contiguous()

    def index(self, p: torch.Tensor):
        vmin = torch.tensor(self.vmin, device=p.device)
        vmax = torch.tensor(self.vmax, device=p.device)
        uv = (p - vmin) / (vmax - vmin)
        uv = uv * torch.tensor(self.res, device=p.device, dtype=p.dtype) + 0.5
        uv = uv.to(torch.int32)
        valid = (uv[:, 0] >= 0) & (uv[:, 0] < self.res[0]) & (uv[:, 1] >= 0) & (uv[:, 1] < self.res[1])
        return valid, uv[:, 0] + (self.res[1] - uv[:, 1]) * self.res[0]


@dataclass
class Intersection:
    valid: torch.Tensor = None
    p: torch.Tensor = None
    n: torch.Tensor = None
    val: torch.Tensor = None
    prim_id: torch.Tensor = None
    t_seg: torch.Tensor = None
    t: torch.Tensor = None
    count: torch.Tensor = None
    J: torch.Tensor = None


@dataclass
class ClosestPointRecord:
    """Boundary record (wos/scene.py:65-82): valid, closest point p, normal n
    (oriented towards the query point, i.e. inward for interior points),
    segment parameter t, boundary value val, primitive prim_id."""
    valid: torch.Tensor = None
    p: torch.Tensor = None
    n: torch.Tensor = None
    t: torch.Tensor = None
    val: torch.Tensor = None
    prim_id: torch.Tensor = None
    J: torch.Tensor = None
    contrib: torch.Tensor = None

    def as_dict(self):
        t = self.t.reshape(-1)
        tuv = torch.stack([t, torch.zeros_like(t)], 1)
        return dict(valid=self.valid.to(torch.uint8), pt=self.p, n=self.n, tuv=tuv, prim=self.prim_id)


@dataclass
class BoundarySamplingRecord:
    p: torch.Tensor = None
    n: torch.Tensor = None
    val: torch.Tensor = None
    prim_id: torch.Tensor = None
    t: torch.Tensor = None
    pdf: torch.Tensor = None


class Polyline:
    """Closed or open 2D polyline boundary with per-vertex Dirichlet values
    (wos/scene.py:192-475; native side include/scene.cuh:316-495).

    vertices (nV, 2), indices (nF, 2) with CCW orientation for a closed curve
    (interior has negative signed distance), values (nV,).  source_type /
    source_params select the analytic source f of -Lap u = f
    (include/scene.cuh:270-301).  use_bvh selects LBVH or brute-force nearest
    queries; both return the same primitive (ties to the lowest index), so it
    only changes speed.
    """

    dim = 2

    def __init__(self, vertices, indices, values, source_type=0, source_params=None, use_bvh=True):
        self.vertices = tensor(vertices, torch.float32).reshape(-1, self.dim)
        self.indices = tensor(indices, torch.int32).reshape(-1, self.dim).contiguous()
        self.values = tensor(values, torch.float32).reshape(-1)
        self.source_type = int(source_type)
        if self.source_type != 0 and source_params is None:
            raise ValueError("source_params required for a source")
        self.source_params = tensor(source_params, torch.float32).reshape(-1) if source_params is not None else None
        self.use_bvh = bool(use_bvh)
        self._native = NativeScene(self.vertices.detach(), self.indices, self.values.detach(), self.source_type,
                                   self.source_params)
        self.normals = self._native.normals()
        info = self._native.info()
        self.aabb = (torch.tensor(list(info.aabb_min)[: self.dim]), torch.tensor(list(info.aabb_max)[: self.dim]))
        self.bvh_nodes = int(info.n_nodes)
        self.bvh_depth = int(info.bvh_depth)
        self.init_dist()

    # ------------------------------------------------------------ construction
    @staticmethod
    def from_vertices(vertices, values, **kw):
        n = len(vertices)
        indices = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
        return Polyline(vertices, indices, values, **kw)

    @staticmethod
    def from_obj(filename, normalize=True, flip_orientation=False, **kw):
        """wos/scene.py:211-240: read an OBJ polyline (`v`, `l`, `c` lines),
        centre it on the vertex mean and scale it to unit radius in double
        precision.  A file without `c` lines gets zero values."""
        from .io import normalize_vertices, read_2d_obj
        V, F, g = read_2d_obj(filename, flip_orientation=flip_orientation)
        V = normalize_vertices(V) if normalize else V.astype(np.float32)
        g = g.astype(np.float32) if len(g) == len(V) else np.zeros(len(V), np.float32)
        return Polyline(V, F.astype(np.int32), g, **kw)

    def update_values(self, values):
        """Replace the Dirichlet values (keeps the geometry and LBVH)."""
        self.values = tensor(values, torch.float32).reshape(-1)
        self._native.update_values(self.values.detach())

    def update_vertices(self, vertices):
        """Move the vertices and rebuild normals, AABB and LBVH."""
        self.vertices = tensor(vertices, torch.float32).reshape(-1, self.dim)
        self._native.update_vertices(self.vertices.detach())
        self.normals = self._native.normals()
        info = self._native.info()
        self.aabb = (torch.tensor(list(info.aabb_min)[: self.dim]), torch.tensor(list(info.aabb_max)[: self.dim]))
        self.init_dist()

    def set_source(self, source_type, source_params=None):
        self.source_type = int(source_type)
        self.source_params = tensor(source_params, torch.float32).reshape(-1) if source_params is not None else None
        self._native.set_source(self.source_type, self.source_params)

    def source_params_tensor(self) -> torch.Tensor:
        if self.source_params is None:
            return torch.zeros(0, device=self.vertices.device)
        return self.source_params

    def init_dist(self):
        f = self.indices.long()
        V = self.vertices.detach()
        self.edge_lengths = torch.linalg.norm(V[f[:, 1]] - V[f[:, 0]], dim=1)

    # ------------------------------------------------------------ queries
    def closest_point_preliminary(self, p) -> torch.Tensor:
        return self._native.closest(points(p, self.dim), self.use_bvh, want=("prim",))["prim"]

    def closest_point(self, p) -> ClosestPointRecord:
        o = self._native.closest(points(p, self.dim), self.use_bvh, want=("prim", "tuv", "pt", "n"))
        its = ClosestPointRecord(valid=o["prim"] >= 0, p=o["pt"], n=o["n"], t=o["tuv"][:, 0].contiguous(),
                                 prim_id=o["prim"])
        its.val = self.dirichlet(its)
        return its

    def sdf(self, p) -> torch.Tensor:
        return self._native.sdf(points(p, self.dim), self.use_bvh)

    def is_inside(self, p) -> torch.Tensor:
        return self._native.closest(points(p, self.dim), self.use_bvh, want=("inside",))["inside"].bool()

    def largest_inscribed_ball(self, its: ClosestPointRecord, epsilon=1e-3) -> torch.Tensor:
        return self._native.inscribed_ball(its.valid.to(torch.uint8), its.p.detach(), its.n.detach(), epsilon,
                                           self.use_bvh)

    def dirichlet(self, its: ClosestPointRecord) -> torch.Tensor:
        """lerp of the segment's vertex values at t (wos/scene.py:353-357);
        attached to `values`."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        va, vb = self.values[f[:, 0]], self.values[f[:, 1]]
        t = its.t.reshape(-1)
        return torch.where(its.valid, va + t * (vb - va), torch.zeros_like(va))

    def source_function(self, p) -> torch.Tensor:
        """f(p) (wos/scene.py:359-381), attached to source_params."""
        p = tensor(p).reshape(-1, 2)
        q = self.source_params
        if self.source_type == 1:
            dx = (p[:, 0] - q[0]) ** 2 / (2.0 * q[2] * q[2])
            dy = (p[:, 1] - q[1]) ** 2 / (2.0 * q[3] * q[3])
            return q[4] * torch.exp(-dx - dy)
        if self.source_type == 2:
            phi = p[:, 0] * q[0] + p[:, 1] * q[1] + q[2]
            return q[3] * torch.sin(phi) + q[4]
        return torch.zeros(p.shape[0], device=p.device)

    def get_point(self, its: ClosestPointRecord) -> ClosestPointRecord:
        """Boundary point re-expressed through the vertices, p = lerp(v0, v1, t)
        with t detached (wos/scene.py:416-433): attached to `vertices`."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        t = its.t.detach().reshape(-1, 1)
        p0, p1 = self.vertices[f[:, 0]], self.vertices[f[:, 1]]
        v0, v1 = self.values[f[:, 0]], self.values[f[:, 1]]
        p = p0 + t * (p1 - p0)
        v = v0 + t[:, 0] * (v1 - v0)
        l = torch.linalg.norm(p1 - p0, dim=1)
        return ClosestPointRecord(valid=its.valid, p=p, n=its.n, t=t[:, 0], val=v, prim_id=its.prim_id,
                                  J=l / l.detach())

    def tangent_derivative(self, its: ClosestPointRecord):
        """Tangential gradient of the boundary data (wos/scene.py:451-460)."""
        prim = its.prim_id.long().clamp_min(0)
        f = self.indices.long()[prim]
        v0, v1 = self.vertices[f[:, 0]].detach(), self.vertices[f[:, 1]].detach()
        val0, val1 = self.values[f[:, 0]].detach(), self.values[f[:, 1]].detach()
        e = v1 - v0
        l = torch.linalg.norm(e, dim=1)
        dv = (val1 - val0) / l
        dt = e / l[:, None]
        return dv * dt[:, 0], dv * dt[:, 1]

    def write_obj(self, filename):
        from .io import write_2d_obj
        write_2d_obj(filename, self.vertices.detach().cpu().numpy(), self.indices.cpu().numpy(),
                     self.values.detach().cpu().numpy())
