"""numpy / ctypes binding of the CPU oracle (oracle/wos_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker and as the timed CPU baseline.
The product package (diff-wos_b200/wos) never imports it.

Parity status: the oracle is pinned by analytic solutions (harmonic and
Poisson known answers), by the reference's own Green's-function CDF table and
by the reference's point-triangle routine (tests/golden/).  The reference
ships no golden walk outputs and cannot run here (Dr.Jit/Mitsuba absent,
lbvh submodule empty), so walk-level parity against the reference itself is
statistical (closed forms), not bitwise.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"


class Params(ctypes.Structure):
    _fields_ = [
        ("nwalks", ctypes.c_int32),
        ("nsteps", ctypes.c_int32),
        ("epsilon", ctypes.c_float),
        ("double_sided", ctypes.c_int32),
        ("prevent_fd_artifacts", ctypes.c_int32),
        ("use_IS_for_greens", ctypes.c_int32),
        ("include_source", ctypes.c_int32),
        ("project_unterminated", ctypes.c_int32),
        ("use_bvh", ctypes.c_int32),
        ("walk_offset", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
        ("jitter", ctypes.c_float * 3),
    ]


class AdjParams(ctypes.Structure):
    _fields_ = [
        ("epsilon2", ctypes.c_float),
        ("clamping", ctypes.c_float),
        ("control_variates", ctypes.c_int32),
        ("source_in_normal_derivative", ctypes.c_int32),
        ("ball_epsilon", ctypes.c_float),
        ("want_dV", ctypes.c_int32),
        ("want_dg", ctypes.c_int32),
        ("want_dsrc", ctypes.c_int32),
    ]


class Detector(ctypes.Structure):
    """Must match wos_detector in include/wos_b200.h."""
    _fields_ = [
        ("vmin", ctypes.c_float * 2),
        ("vmax", ctypes.c_float * 2),
        ("res", ctypes.c_int32 * 2),
        ("axis_u", ctypes.c_int32),
        ("axis_v", ctypes.c_int32),
        ("slab_axis", ctypes.c_int32),
        ("slab_center", ctypes.c_float),
        ("slab_half_width", ctypes.c_float),
        ("size", ctypes.c_float),
        ("flags", ctypes.c_int32),
    ]


def make_detector(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(8, 8), axis_u=0, axis_v=1, slab_axis=-1, slab_center=0.0,
                  slab_half_width=0.0, size=None, flags=0) -> Detector:
    if size is None:
        size = (vmax[0] - vmin[0]) * (vmax[1] - vmin[1]) * (2 * slab_half_width if slab_axis >= 0 else 1.0)
    return Detector((ctypes.c_float * 2)(*vmin), (ctypes.c_float * 2)(*vmax), (ctypes.c_int32 * 2)(*res),
                    int(axis_u), int(axis_v), int(slab_axis), float(slab_center), float(slab_half_width), float(size),
                    int(flags))


def make_params(nwalks=1, nsteps=32, epsilon=1e-3, double_sided=False, prevent_fd_artifacts=False,
                use_IS_for_greens=False, include_source=False, project_unterminated=False, use_bvh=True,
                walk_offset=0, seed=0, jitter=(0.0, 0.0, 0.0)) -> Params:
    j = tuple(float(x) for x in jitter) + (0.0,) * (3 - len(jitter))
    return Params(int(nwalks), int(nsteps), float(epsilon), int(double_sided), int(prevent_fd_artifacts),
                  int(use_IS_for_greens), int(include_source), int(project_unterminated), int(use_bvh),
                  int(walk_offset), int(seed), (ctypes.c_float * 3)(*j[:3]))


def make_adj(epsilon2=1e-3, clamping=1e-1, control_variates=True, source_in_normal_derivative=False,
             ball_epsilon=1e-3, want_dV=True, want_dg=True, want_dsrc=True) -> AdjParams:
    return AdjParams(float(epsilon2), float(clamping), int(control_variates), int(source_in_normal_derivative),
                     float(ball_epsilon), int(want_dV), int(want_dg), int(want_dsrc))


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        I = ctypes.c_int
        L.orc_scene_create.restype = P
        L.orc_scene_create.argtypes = [I, P, I, P, I, P, I, P]
        L.orc_scene_destroy.argtypes = [P]
        L.orc_scene_normals.argtypes = [P, P]
        L.orc_scene_aabb.argtypes = [P, P]
        L.orc_g_cdf.argtypes = [P, I]
        L.orc_bvh_export.restype = I
        L.orc_bvh_export.argtypes = [P, P, P]
        L.orc_closest.argtypes = [P, P, I, I, P, P, P, P, P, P, P, I]
        L.orc_bvh_counts.argtypes = [P, P, I, P, P, I]
        L.orc_inscribed_ball.argtypes = [P, P, P, P, I, ctypes.c_float, I, P, I]
        L.orc_walk_values.argtypes = [P, P, I, ctypes.POINTER(Params), P, P, P, I]
        L.orc_solve_f64_2d.argtypes = [P, P, I, I, I, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, I, P, P, P]
        L.orc_walk_records.argtypes = [P, P, I, ctypes.POINTER(Params), P, P, P, P, P, P, I]
        L.orc_reduce.argtypes = [P, I, I, P, P]
        L.orc_normal_derivative.argtypes = [P, P, P, P, P, P, I, ctypes.POINTER(Params), ctypes.POINTER(AdjParams),
                                            P, I]
        L.orc_adjoint.argtypes = [P, P, I, ctypes.POINTER(Params), ctypes.POINTER(AdjParams), P, P, P, P, I]
        L.orc_math.argtypes = [I, P, P, P, I]
        L.orc_philox.argtypes = [ctypes.c_uint64, P, P, I]
        L.orc_tri_closest.argtypes = [P, P, P, P, I, P, P]
        L.orc_walk_counted.argtypes = [P, P, I, ctypes.POINTER(Params), P, I, P]
        L.orc_soft_walk.argtypes = [P, P, I, ctypes.POINTER(Params), P, I]
        L.orc_adjoint_counted.argtypes = [P, P, I, ctypes.POINTER(Params), ctypes.POINTER(AdjParams), P, P, P, P, I,
                                          P]
        L.orc_normal_derivative_r.argtypes = [P, P, P, P, P, P, P, I, ctypes.POINTER(Params),
                                              ctypes.POINTER(AdjParams), P, I]
        L.orc_boundary_term.argtypes = [P, ctypes.POINTER(Detector), I, ctypes.c_uint64, P, P, P, P, I]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OracleScene:
    """A scene in the oracle: vertices (nV x dim), faces (nF x dim), values (nV)."""

    def __init__(self, V, F, g, source_type=0, source_params=None):
        self.V = _f32(V)
        self.F = _i32(F)
        self.g = _f32(g)
        self.dim = self.V.shape[1]
        self.src = _f32(source_params if source_params is not None else np.zeros(5))
        self.source_type = int(source_type)
        self.h = lib().orc_scene_create(self.dim, _p(self.V), self.V.shape[0], _p(self.F), self.F.shape[0],
                                        _p(self.g), self.source_type, _p(self.src))

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().orc_scene_destroy(self.h)
            except TypeError:  # module globals already torn down at interpreter exit
                pass
            self.h = None

    def normals(self):
        out = np.zeros_like(self.V)
        lib().orc_scene_normals(self.h, _p(out))
        return out

    def aabb(self):
        out = np.zeros(2 * self.dim, np.float32)
        lib().orc_scene_aabb(self.h, _p(out))
        return out[: self.dim], out[self.dim:]

    def bvh(self):
        nF = self.F.shape[0]
        ch = np.zeros((max(nF - 1, 1), 2), np.int32)
        keys = np.zeros(nF, np.uint64)
        n = lib().orc_bvh_export(self.h, _p(ch), _p(keys))
        return ch[:n], keys

    def closest(self, P, use_bvh=True, nthreads=0):
        P = _f32(P)
        n = P.shape[0]
        out = dict(prim=np.zeros(n, np.int32), dist=np.zeros(n, np.float32), tuv=np.zeros((n, 2), np.float32),
                   pt=np.zeros((n, self.dim), np.float32), n=np.zeros((n, self.dim), np.float32),
                   sdf=np.zeros(n, np.float32), inside=np.zeros(n, np.uint8))
        lib().orc_closest(self.h, _p(P), n, int(use_bvh), _p(out["prim"]), _p(out["dist"]), _p(out["tuv"]),
                          _p(out["pt"]), _p(out["n"]), _p(out["sdf"]), _p(out["inside"]), nthreads)
        return out

    def bvh_counts(self, P, nthreads=0):
        P = _f32(P)
        n = P.shape[0]
        nb = np.zeros(n, np.int32)
        npr = np.zeros(n, np.int32)
        lib().orc_bvh_counts(self.h, _p(P), n, _p(nb), _p(npr), nthreads)
        return nb, npr

    def inscribed_ball(self, valid, pt, nrm, eps=1e-3, use_bvh=True, nthreads=0):
        valid = np.ascontiguousarray(valid, np.uint8)
        pt, nrm = _f32(pt), _f32(nrm)
        R = np.zeros(valid.shape[0], np.float32)
        lib().orc_inscribed_ball(self.h, _p(pt), _p(nrm), _p(valid), valid.shape[0], eps, int(use_bvh), _p(R),
                                 nthreads)
        return R

    def solve_f64(self, P, nwalks, fconst=0.0, eps=1e-3, max_steps=100_000, seed=0, nthreads=0):
        """FP64 reference solution of -lap u = fconst with this scene's g (2D):
        per-point mean and variance over `nwalks` double-precision walks whose
        source term is its expectation f R^2 / 4 per step.  Returns (mean,
        var, truncated walk count)."""
        assert self.dim == 2
        P = np.ascontiguousarray(P, dtype=np.float64)
        n = P.shape[0]
        mean = np.zeros(n, np.float64)
        var = np.zeros(n, np.float64)
        tr = ctypes.c_longlong(0)
        lib().orc_solve_f64_2d(self.h, _p(P), n, int(nwalks), int(max_steps), float(eps), float(fconst),
                               int(seed) & 0xFFFFFFFFFFFFFFFF, nthreads, _p(mean), _p(var), ctypes.byref(tr))
        return mean, var, int(tr.value)

    def walk_values(self, P, params: Params, nthreads=0):
        P = _f32(P)
        n = P.shape[0]
        vals = np.zeros((n, params.nwalks), np.float32)
        valid = np.zeros((n, params.nwalks), np.uint8)
        steps = np.zeros((n, params.nwalks), np.int32)
        lib().orc_walk_values(self.h, _p(P), n, ctypes.byref(params), _p(vals), _p(valid), _p(steps), nthreads)
        return vals, valid, steps

    def walk_records(self, P, params: Params, nthreads=0):
        P = _f32(P)
        n = P.shape[0]
        out = dict(valid=np.zeros(n, np.uint8), pt=np.zeros((n, self.dim), np.float32),
                   n=np.zeros((n, self.dim), np.float32), tuv=np.zeros((n, 2), np.float32),
                   prim=np.zeros(n, np.int32), contrib=np.zeros(n, np.float32))
        lib().orc_walk_records(self.h, _p(P), n, ctypes.byref(params), _p(out["valid"]), _p(out["pt"]),
                               _p(out["n"]), _p(out["tuv"]), _p(out["prim"]), _p(out["contrib"]), nthreads)
        return out

    def normal_derivative(self, rec, params: Params, adj: AdjParams, nthreads=0, R=None):
        """One estimate per record; R: per-record ball radii (override_R)."""
        n = rec["valid"].shape[0]
        out = np.zeros((n, self.dim), np.float32)
        Rv = None if R is None else np.ascontiguousarray(np.broadcast_to(np.asarray(R, np.float32), (n,)))
        lib().orc_normal_derivative_r(self.h, _p(np.ascontiguousarray(rec["valid"], np.uint8)), _p(_f32(rec["pt"])),
                                      _p(_f32(rec["n"])), _p(_f32(rec["tuv"])), _p(_i32(rec["prim"])), _p(Rv), n,
                                      ctypes.byref(params), ctypes.byref(adj), _p(out), nthreads)
        return out

    def adjoint(self, P, params: Params, adj: AdjParams, dLdu, nthreads=0):
        P = _f32(P)
        dLdu = _f32(dLdu)
        dV = np.zeros(self.V.shape, np.float64)
        dg = np.zeros(self.V.shape[0], np.float64)
        ds = np.zeros(5, np.float64)
        lib().orc_adjoint(self.h, _p(P), P.shape[0], ctypes.byref(params), ctypes.byref(adj), _p(dLdu), _p(dV),
                          _p(dg), _p(ds), nthreads)
        return dV, dg, ds


    def boundary_term(self, det: Detector, nwalks, seed=0, dV_dir=None, dLdI=None, nthreads=0):
        """WoSBoundary's image-space boundary term: the derivative image for
        vertex motion dV_dir and / or the vertex gradient of pixel weights
        dLdI (both float64)."""
        npix = int(det.res[0]) * int(det.res[1])
        tV = _f32(dV_dir) if dV_dir is not None else None
        w = _f32(dLdI) if dLdI is not None else None
        img = np.zeros(npix, np.float64) if tV is not None else None
        dV = np.zeros(self.V.shape, np.float64) if w is not None else None
        lib().orc_boundary_term(self.h, ctypes.byref(det), int(nwalks), int(seed) & 0xFFFFFFFFFFFFFFFF, _p(tV),
                                _p(img), _p(w), _p(dV), nthreads)
        return img, dV

    def soft_walk(self, P, params: Params, nthreads=0):
        """Per-walk values of the soft-edge walk (Baseline), points x walks."""
        P = _f32(P)
        n = P.shape[0]
        vals = np.zeros((n, params.nwalks), np.float32)
        lib().orc_soft_walk(self.h, _p(P), n, ctypes.byref(params), _p(vals), nthreads)
        return vals

    def walk_counted(self, P, params: Params, nthreads=0):
        """Per-walk values plus LBVH work totals {queries, node visits, prims}."""
        P = _f32(P)
        n = P.shape[0]
        vals = np.zeros((n, params.nwalks), np.float32)
        counts = np.zeros(3, np.int64)
        lib().orc_walk_counted(self.h, _p(P), n, ctypes.byref(params), _p(vals), nthreads, _p(counts))
        return vals, dict(queries=int(counts[0]), nodes=int(counts[1]), prims=int(counts[2]))

    def adjoint_counted(self, P, params: Params, adj: AdjParams, dLdu, nthreads=0):
        P = _f32(P)
        dLdu = _f32(dLdu)
        dV = np.zeros(self.V.shape, np.float64)
        dg = np.zeros(self.V.shape[0], np.float64)
        ds = np.zeros(5, np.float64)
        counts = np.zeros(3, np.int64)
        lib().orc_adjoint_counted(self.h, _p(P), P.shape[0], ctypes.byref(params), ctypes.byref(adj), _p(dLdu),
                                  _p(dV), _p(dg), _p(ds), nthreads, _p(counts))
        return (dV, dg, ds), dict(queries=int(counts[0]), nodes=int(counts[1]), prims=int(counts[2]))


def reduce(vals):
    vals = _f32(vals)
    n, nw = vals.shape
    mean = np.zeros(n, np.float64)
    var = np.zeros(n, np.float64)
    lib().orc_reduce(_p(vals), n, nw, _p(mean), _p(var))
    return mean, var


def g_cdf(n=10000):
    out = np.zeros(n, np.float32)
    lib().orc_g_cdf(_p(out), n)
    return out


def math_fn(which: str, x, y=None):
    codes = {"sincos_2pi": 0, "sin": 1, "cos": 2, "log": 3, "exp": 4, "atan2": 5}
    x = _f32(x)
    y = _f32(y) if y is not None else np.zeros_like(x)
    out = np.zeros(x.shape[0] * (2 if which == "sincos_2pi" else 1), np.float32)
    lib().orc_math(codes[which], _p(x), _p(y), _p(out), x.shape[0])
    return out.reshape(-1, 2) if which == "sincos_2pi" else out


def tri_closest(A, B, C, P):
    """(uv = (w_b, w_c), distance) of points P to triangles (A, B, C)."""
    A, B, C, P = _f32(A), _f32(B), _f32(C), _f32(P)
    n = P.shape[0]
    uv = np.zeros((n, 2), np.float32)
    d = np.zeros(n, np.float32)
    lib().orc_tri_closest(_p(A), _p(B), _p(C), _p(P), n, _p(uv), _p(d))
    return uv, d


def philox(seed: int, ctr):
    ctr = np.ascontiguousarray(ctr, np.uint32)
    out = np.zeros_like(ctr)
    lib().orc_philox(seed, _p(ctr), _p(out), ctr.shape[0])
    return out
