"""Thin torch-facing wrapper of the C ABI: one NativeScene per scene.

Every method takes and returns torch CUDA tensors and runs on the current
torch stream.  This is the only module that calls libwos_b200.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import WosAdjointParams, WosParams, call


def cuda_device() -> torch.device:
    if not torch.cuda.is_available():
        raise _lib.WosError(_lib.WOS_ERR_UNSUPPORTED, "a CUDA device is required (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def as_cuda(x, dtype, shape_last=None) -> torch.Tensor:
    """Contiguous CUDA tensor of dtype (detached copy only when needed)."""
    if isinstance(x, torch.Tensor):
        t = x.detach()
        if t.device.type != "cuda" or t.dtype != dtype:
            t = t.to(device=cuda_device(), dtype=dtype)
    else:
        t = torch.as_tensor(np.asarray(x), dtype=dtype, device=cuda_device())
    t = t.contiguous()
    if shape_last is not None and t.dim() == 1 and t.numel() % shape_last == 0 and shape_last > 1:
        t = t.view(-1, shape_last)
    return t


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


@dataclass
class WalkSettings:
    nwalks: int = 1
    nsteps: int = 32
    epsilon: float = 1e-3
    double_sided: bool = False
    prevent_fd_artifacts: bool = False
    use_IS_for_greens: bool = False
    include_source: bool = False
    project_unterminated: bool = False
    use_bvh: bool = True
    walk_offset: int = 0
    seed: int = 0
    jitter: tuple = (0.0, 0.0, 0.0)  # start-point jitter extent per axis (pixel sampling)

    def c(self) -> WosParams:
        j = tuple(float(x) for x in self.jitter) + (0.0,) * (3 - len(self.jitter))
        return WosParams(int(self.nwalks), int(self.nsteps), float(self.epsilon), int(self.double_sided),
                         int(self.prevent_fd_artifacts), int(self.use_IS_for_greens), int(self.include_source),
                         int(self.project_unterminated), int(self.use_bvh), int(self.walk_offset) & 0xFFFFFFFF,
                         int(self.seed) & 0xFFFFFFFFFFFFFFFF, (ctypes.c_float * 3)(*j[:3]))


@dataclass
class AdjointSettings:
    epsilon2: float = 1e-3
    clamping: float = 1e-1
    control_variates: bool = True
    source_in_normal_derivative: bool = True
    ball_epsilon: float = 1e-3
    want_dV: bool = True
    want_dg: bool = False
    want_dsrc: bool = False

    def c(self) -> WosAdjointParams:
        return WosAdjointParams(float(self.epsilon2), float(self.clamping), int(self.control_variates),
                                int(self.source_in_normal_derivative), float(self.ball_epsilon), int(self.want_dV),
                                int(self.want_dg), int(self.want_dsrc))


class NativeScene:
    """Owns a wos_scene_t built from vertices (nV x dim), faces (nF x dim) and
    Dirichlet values (nV)."""

    def __init__(self, V, F, g, source_type: int = 0, source_params=None):
        V = as_cuda(V, torch.float32)
        F = as_cuda(F, torch.int32)
        g = as_cuda(g, torch.float32).reshape(-1)
        if V.dim() != 2 or V.shape[1] not in (2, 3):
            raise ValueError("vertices must be (nV, 2) or (nV, 3)")
        if F.dim() != 2 or F.shape[1] != V.shape[1]:
            raise ValueError("indices must be (nF, dim)")
        if g.numel() != V.shape[0]:
            raise ValueError("values must have one entry per vertex")
        self.dim = int(V.shape[1])
        self.nV = int(V.shape[0])
        self.nF = int(F.shape[0])
        src = None
        if source_type:
            src = (ctypes.c_float * 5)(*[float(v) for v in _host5(source_params)])
        h = ctypes.c_void_p()
        call("wos_scene_create", self.dim, V.data_ptr(), self.nV, F.data_ptr(), self.nF, g.data_ptr(),
             int(source_type), ctypes.cast(src, ctypes.c_void_p) if src is not None else None, stream(),
             ctypes.byref(h))
        self.h = h
        self.device = V.device

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            try:
                _lib.lib().wos_scene_destroy(self.h, stream())
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.close()

    # ------------------------------------------------------------ scene
    def info(self) -> _lib.WosSceneInfo:
        i = _lib.WosSceneInfo()
        call("wos_scene_get_info", self.h, ctypes.byref(i))
        return i

    def normals(self) -> torch.Tensor:
        out = torch.empty((self.nV, self.dim), dtype=torch.float32, device=self.device)
        call("wos_scene_get_normals", self.h, out.data_ptr(), stream())
        return out

    def update_values(self, g):
        g = as_cuda(g, torch.float32).reshape(-1)
        if g.numel() != self.nV:
            raise ValueError("values must have one entry per vertex")
        call("wos_scene_update_values", self.h, g.data_ptr(), stream())
        self._keep = g  # keep alive until the copy has run

    def update_vertices(self, V):
        V = as_cuda(V, torch.float32)
        if tuple(V.shape) != (self.nV, self.dim):
            raise ValueError("vertices must keep their shape")
        call("wos_scene_update_vertices", self.h, V.data_ptr(), stream())

    def set_source(self, source_type: int, params):
        src = (ctypes.c_float * 5)(*[float(v) for v in _host5(params)]) if source_type else None
        call("wos_scene_set_source", self.h, int(source_type), ctypes.cast(src, ctypes.c_void_p) if src else None)

    # ------------------------------------------------------------ queries
    def closest(self, P, use_bvh=True, want=("prim", "dist", "tuv", "pt", "n", "sdf", "inside")):
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        out = {}
        specs = dict(prim=((n,), torch.int32), dist=((n,), torch.float32), tuv=((n, 2), torch.float32),
                     pt=((n, self.dim), torch.float32), n=((n, self.dim), torch.float32),
                     sdf=((n,), torch.float32), inside=((n,), torch.uint8))
        for k in want:
            shp, dt = specs[k]
            out[k] = torch.empty(shp, dtype=dt, device=d)
        if n:
            call("wos_closest_point", self.h, P.data_ptr(), n, int(use_bvh), _ptr(out.get("prim")),
                 _ptr(out.get("dist")), _ptr(out.get("tuv")), _ptr(out.get("pt")), _ptr(out.get("n")),
                 _ptr(out.get("sdf")), _ptr(out.get("inside")), stream())
        return out

    def sdf(self, P, use_bvh=True) -> torch.Tensor:
        """Signed distance to the boundary, negative inside (wos_sdf)."""
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        if n:
            call("wos_sdf", self.h, P.data_ptr(), n, int(use_bvh), out.data_ptr(), stream())
        return out

    def inscribed_ball(self, valid, pt, nrm, epsilon=1e-3, use_bvh=True) -> torch.Tensor:
        valid = as_cuda(valid, torch.uint8).reshape(-1)
        pt = as_cuda(pt, torch.float32, self.dim)
        nrm = as_cuda(nrm, torch.float32, self.dim)
        n = int(valid.numel())
        R = torch.empty(n, dtype=torch.float32, device=self.device)
        if n:
            call("wos_largest_inscribed_ball", self.h, valid.data_ptr(), pt.data_ptr(), nrm.data_ptr(), n,
                 float(epsilon), int(use_bvh), R.data_ptr(), stream())
        return R

    # ------------------------------------------------------------ walks
    def records(self, P, s: WalkSettings):
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        out = dict(valid=torch.empty(n, dtype=torch.uint8, device=d),
                   pt=torch.empty((n, self.dim), dtype=torch.float32, device=d),
                   n=torch.empty((n, self.dim), dtype=torch.float32, device=d),
                   tuv=torch.empty((n, 2), dtype=torch.float32, device=d),
                   prim=torch.empty(n, dtype=torch.int32, device=d),
                   contrib=torch.empty(n, dtype=torch.float32, device=d))
        if n:
            c = s.c()
            call("wos_walk_records", self.h, P.data_ptr(), n, ctypes.byref(c), out["valid"].data_ptr(),
                 out["pt"].data_ptr(), out["n"].data_ptr(), out["tuv"].data_ptr(), out["prim"].data_ptr(),
                 out["contrib"].data_ptr(), stream())
        return out

    def values(self, P, s: WalkSettings, want_steps=False, plain=False):
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        vals = torch.empty((n, s.nwalks), dtype=torch.float32, device=self.device)
        steps = torch.empty((n, s.nwalks), dtype=torch.int32, device=self.device) if want_steps else None
        if n:
            c = s.c()
            if plain:
                call("wos_walk_values_plain", self.h, P.data_ptr(), n, ctypes.byref(c), vals.data_ptr(), stream())
            else:
                call("wos_walk_values", self.h, P.data_ptr(), n, ctypes.byref(c), vals.data_ptr(), _ptr(steps),
                     stream())
        return (vals, steps) if want_steps else vals

    def solve(self, P, s: WalkSettings, want_var=False, workspace: torch.Tensor | None = None):
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        mean = torch.empty(n, dtype=torch.float64, device=self.device)
        var = torch.empty(n, dtype=torch.float64, device=self.device) if want_var else None
        if n:
            c = s.c()
            need = _lib.lib().wos_solve_workspace_size(n, ctypes.byref(c))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
            call("wos_solve", self.h, P.data_ptr(), n, ctypes.byref(c), mean.data_ptr(), _ptr(var),
                 workspace.data_ptr(), need, stream())
        return (mean, var) if want_var else mean

    def solve_records(self, P, s: WalkSettings, want_dcontrib=False, want_var=False,
                      workspace: torch.Tensor | None = None):
        """solve() that keeps each walk's boundary record (and, optionally, its
        source-parameter derivative) for adjoint_records()."""
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        mean = torch.empty(n, dtype=torch.float64, device=d)
        var = torch.empty(n, dtype=torch.float64, device=d) if want_var else None
        rb = _lib.lib().wos_walk_record_bytes(self.dim)
        rec = torch.empty(max(n * s.nwalks * rb, 1), dtype=torch.uint8, device=d)
        dc = torch.empty(max(n * s.nwalks * 5, 1), dtype=torch.float32, device=d) if want_dcontrib else None
        if n:
            c = s.c()
            need = _lib.lib().wos_solve_workspace_size(n, ctypes.byref(c))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_solve_records", self.h, P.data_ptr(), n, ctypes.byref(c), mean.data_ptr(), _ptr(var),
                 rec.data_ptr(), _ptr(dc), workspace.data_ptr(), need, stream())
        return mean, var, rec, dc

    def adjoint_records(self, P, s: WalkSettings, a: AdjointSettings, dLdu, rec, dc,
                        workspace: torch.Tensor | None = None):
        P = as_cuda(P, torch.float32, self.dim)
        dLdu = as_cuda(dLdu, torch.float32).reshape(-1)
        n = int(P.shape[0])
        d = self.device
        dV = torch.zeros((self.nV, self.dim), dtype=torch.float32, device=d) if a.want_dV else None
        dg = torch.zeros(self.nV, dtype=torch.float32, device=d) if a.want_dg else None
        ds = torch.zeros(5, dtype=torch.float32, device=d) if a.want_dsrc else None
        if n:
            c, ca = s.c(), a.c()
            need = _lib.lib().wos_adjoint_records_workspace_size(self.h, n, ctypes.byref(c))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_adjoint_records", self.h, P.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca), dLdu.data_ptr(),
                 rec.data_ptr(), _ptr(dc), _ptr(dV), _ptr(dg), _ptr(ds), workspace.data_ptr(), need, stream())
        return dV, dg, ds

    def solve_adjoint(self, P, s: WalkSettings, a: AdjointSettings, loss_kind=1, target=None, want_var=False,
                      workspace: torch.Tensor | None = None):
        """Fused forward + adjoint of a pointwise loss of the means (loss_kind
        1: mean(u^2), 2: mean((u - target)^2), 0: target holds dL/du)."""
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        tg = as_cuda(target, torch.float32).reshape(-1) if target is not None else None
        mean = torch.empty(n, dtype=torch.float64, device=d)
        var = torch.empty(n, dtype=torch.float64, device=d) if want_var else None
        loss = torch.zeros(1, dtype=torch.float64, device=d)
        dV = torch.zeros((self.nV, self.dim), dtype=torch.float32, device=d) if a.want_dV else None
        dg = torch.zeros(self.nV, dtype=torch.float32, device=d) if a.want_dg else None
        ds = torch.zeros(5, dtype=torch.float32, device=d) if a.want_dsrc else None
        if n:
            c, ca = s.c(), a.c()
            need = _lib.lib().wos_solve_adjoint_workspace_size(self.h, n, ctypes.byref(c), ctypes.byref(ca))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_solve_adjoint", self.h, P.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca), int(loss_kind),
                 _ptr(tg), mean.data_ptr(), _ptr(var), loss.data_ptr(), _ptr(dV), _ptr(dg), _ptr(ds),
                 workspace.data_ptr(), need, stream())
        return dict(mean=mean, var=var, loss=loss, dV=dV, dg=dg, dsrc=ds)

    def solve_tangent(self, P, s: WalkSettings, a: AdjointSettings, dV=None, dg=None, dsrc=None, want_var=False,
                      workspace: torch.Tensor | None = None):
        """Fused forward solve + forward-mode derivative of the per-point means
        along the direction (dV: nV x dim, dg: nV, dsrc: 5; None = still)."""
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        mean = torch.empty(n, dtype=torch.float64, device=d)
        tan = torch.empty(n, dtype=torch.float64, device=d)
        var = torch.empty(n, dtype=torch.float64, device=d) if want_var else None
        tvar = torch.empty(n, dtype=torch.float64, device=d) if want_var else None
        tV = as_cuda(dV, torch.float32, self.dim) if dV is not None else None
        if tV is not None and tV.shape[0] != self.nV:
            raise ValueError("dV must be nV x dim")
        tg = as_cuda(dg, torch.float32).reshape(-1) if dg is not None else None
        if tg is not None and tg.numel() != self.nV:
            raise ValueError("dg must have one entry per vertex")
        ts = as_cuda(dsrc, torch.float32).reshape(-1) if dsrc is not None else None
        if ts is not None and ts.numel() != 5:
            raise ValueError("dsrc must have 5 entries")
        if n:
            c, ca = s.c(), a.c()
            need = _lib.lib().wos_solve_tangent_workspace_size(self.h, n, ctypes.byref(c), ctypes.byref(ca))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_solve_tangent", self.h, P.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca), _ptr(tV), _ptr(tg),
                 _ptr(ts), mean.data_ptr(), _ptr(var), tan.data_ptr(), _ptr(tvar), workspace.data_ptr(), need,
                 stream())
        return dict(mean=mean, var=var, tangent=tan, tangent_var=tvar)

    def soft_walk(self, P, s: WalkSettings, dV=None, dg=None, want_tangent=False, want_var=False):
        """Soft-edge walk (wos_soft_walk): per-point mean of the walk values
        and, with want_tangent, of their derivatives along (dV, dg)."""
        P = as_cuda(P, torch.float32, self.dim)
        n = int(P.shape[0])
        d = self.device
        mean = torch.empty(n, dtype=torch.float64, device=d)
        var = torch.empty(n, dtype=torch.float64, device=d) if want_var else None
        tan = torch.empty(n, dtype=torch.float64, device=d) if want_tangent else None
        tvar = torch.empty(n, dtype=torch.float64, device=d) if (want_tangent and want_var) else None
        tV = as_cuda(dV, torch.float32, self.dim) if dV is not None else None
        tg = as_cuda(dg, torch.float32).reshape(-1) if dg is not None else None
        if n:
            c = s.c()
            need = _lib.lib().wos_soft_walk_workspace_size(n, ctypes.byref(c))
            ws = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_soft_walk", self.h, P.data_ptr(), n, ctypes.byref(c), _ptr(tV), _ptr(tg), mean.data_ptr(),
                 _ptr(var), _ptr(tan), _ptr(tvar), ws.data_ptr(), need, stream())
        return dict(mean=mean, var=var, tangent=tan, tangent_var=tvar)

    def soft_walk_adjoint(self, P, s: WalkSettings, dLdu, want_dV=True, want_dg=True):
        """Reverse mode of the soft-edge walk (wos_soft_walk_adjoint): the
        gradients of sum_i dLdu[i] mean_i with respect to the vertices and the
        values (None where not wanted)."""
        P = as_cuda(P, torch.float32, self.dim)
        dLdu = as_cuda(dLdu, torch.float32).reshape(-1)
        n = int(P.shape[0])
        if dLdu.numel() != n:
            raise ValueError("dLdu must have one entry per point")
        d = self.device
        dV = torch.zeros((self.nV, self.dim), dtype=torch.float32, device=d) if want_dV else None
        dg = torch.zeros(self.nV, dtype=torch.float32, device=d) if want_dg else None
        if n and (want_dV or want_dg):
            c = s.c()
            call("wos_soft_walk_adjoint", self.h, P.data_ptr(), n, ctypes.byref(c), dLdu.data_ptr(), _ptr(dV),
                 _ptr(dg), stream())
        return dV, dg

    def boundary_term(self, det, nwalks: int, seed: int = 0, dV_dir=None, dLdI=None):
        """Image-space boundary term (wos_boundary_term): the derivative image
        for vertex motion dV_dir (forward mode) and / or the vertex gradient
        of pixel weights dLdI (reverse mode).  `det` is a WosDetector.
        Returns (image_tangent or None, dV or None)."""
        npix = int(det.res[0]) * int(det.res[1])
        d = self.device
        tV = as_cuda(dV_dir, torch.float32, self.dim) if dV_dir is not None else None
        if tV is not None and tV.shape[0] != self.nV:
            raise ValueError("dV_dir must be nV x dim")
        w = as_cuda(dLdI, torch.float32).reshape(-1) if dLdI is not None else None
        if w is not None and w.numel() != npix:
            raise ValueError("dLdI must have one entry per pixel")
        img = torch.zeros(npix, dtype=torch.float64, device=d) if tV is not None else None
        dV = torch.zeros((self.nV, self.dim), dtype=torch.float32, device=d) if w is not None else None
        call("wos_boundary_term", self.h, ctypes.byref(det), int(nwalks), int(seed) & 0xFFFFFFFFFFFFFFFF, _ptr(tV),
             _ptr(img), _ptr(w), _ptr(dV), stream())
        return img, dV

    def normal_derivative(self, rec, s: WalkSettings, a: AdjointSettings, R=None) -> torch.Tensor:
        """One normal-derivative estimate per record (grad * outward normal);
        R: per-record ball radii (override_R), default the inscribed ball."""
        valid = as_cuda(rec["valid"], torch.uint8).reshape(-1)
        n = int(valid.numel())
        out = torch.empty((n, self.dim), dtype=torch.float32, device=self.device)
        if n:
            pt = as_cuda(rec["pt"], torch.float32, self.dim)
            nrm = as_cuda(rec["n"], torch.float32, self.dim)
            tuv = as_cuda(rec["tuv"], torch.float32, 2)
            prim = as_cuda(rec["prim"], torch.int32).reshape(-1)
            c, ca = s.c(), a.c()
            if R is None:
                call("wos_normal_derivative", self.h, valid.data_ptr(), pt.data_ptr(), nrm.data_ptr(),
                     tuv.data_ptr(), prim.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca), out.data_ptr(), stream())
            else:
                Rt = as_cuda(R, torch.float32).reshape(-1)
                if Rt.numel() == 1:
                    Rt = Rt.expand(n).contiguous()
                if Rt.numel() != n:
                    raise ValueError("R must be a scalar or have one entry per record")
                call("wos_normal_derivative_radius", self.h, valid.data_ptr(), pt.data_ptr(), nrm.data_ptr(),
                     tuv.data_ptr(), prim.data_ptr(), Rt.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca),
                     out.data_ptr(), stream())
        return out

    def adjoint(self, P, s: WalkSettings, a: AdjointSettings, dLdu, workspace: torch.Tensor | None = None):
        P = as_cuda(P, torch.float32, self.dim)
        dLdu = as_cuda(dLdu, torch.float32).reshape(-1)
        n = int(P.shape[0])
        if dLdu.numel() != n:
            raise ValueError("dLdu must have one entry per point")
        d = self.device
        dV = torch.zeros((self.nV, self.dim), dtype=torch.float32, device=d) if a.want_dV else None
        dg = torch.zeros(self.nV, dtype=torch.float32, device=d) if a.want_dg else None
        ds = torch.zeros(5, dtype=torch.float32, device=d) if a.want_dsrc else None
        if n:
            c, ca = s.c(), a.c()
            need = _lib.lib().wos_adjoint_workspace_size(self.h)
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(need, dtype=torch.uint8, device=d)
            call("wos_adjoint", self.h, P.data_ptr(), n, ctypes.byref(c), ctypes.byref(ca), dLdu.data_ptr(),
                 _ptr(dV), _ptr(dg), _ptr(ds), workspace.data_ptr(), need, stream())
        return dV, dg, ds


def _host5(params) -> list[float]:
    if params is None:
        return [0.0] * 5
    if isinstance(params, torch.Tensor):
        params = params.detach().cpu().reshape(-1).tolist()
    params = [float(v) for v in np.asarray(params, dtype=np.float64).reshape(-1)]
    if len(params) != 5:
        raise ValueError("source_params must have 5 entries")
    return params
