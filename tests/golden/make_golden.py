"""Generate the golden fixtures in tests/golden/ from the reference sources.

Run, in a checkout where the reference repository is available, with its
path as the one required argument:

    python tests/golden/make_golden.py /path/to/diff-wos [--only NAME ...]

It writes
  g_cdf_ref.json       entries of the reference's tabulated Green's-function
                       CDF (include/tabulated_G_cdf.cuh), read as text;
  ericson_ref.npz      outputs of the reference's point-triangle routine
                       closest_point_triangle (wos/utils.py:108-173);
  meshes/*.obj         the reference's sample meshes (data/meshes), copied
                       as data, and meshes_ref.npz: what the reference's own
                       readers (wos/io.py:20-38 read_2d_obj, :54-71
                       read_3d_obj; wos/scene.py:211-240 Polyline.from_obj)
                       return for them;
  ref_estimators.npz   per-point means and variances of the reference's own
                       Python estimators, executed on small scenes (see
                       make_estimators below).

Everything the reference computes here runs the reference's own Python
modules, loaded from the given path on top of tests/golden/drjit_np.py, a
numpy stand-in for the Dr.Jit / Mitsuba API (neither is installable here).
The reference's C++ extension wos_ext cannot run; the few members of it that
those modules call (the scene constructor's vertex normals and bounding box,
largest_inscribed_ball) are restated in fake_wos_ext below from
include/scene.cuh.  The tests only read the written files; nothing at test
time touches the reference.
"""
from __future__ import annotations

import argparse
import ast
import importlib
import importlib.util
import json
import re
import shutil
import sys
import time
import types
import warnings
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(OUT))
import drjit_np as D  # noqa: E402

REPO = OUT.parent.parent


# ---------------------------------------------------------------- the reference on the stand-in
def fake_wos_ext():
    """The members of the reference's pybind module wos_ext
    (src/python/main.cpp:9-17, src/python/scene.cu:10-88) that its Python
    estimators call, restated from include/scene.cuh."""
    m = types.ModuleType("wos_ext")

    class ClosestPointRecord:
        def __init__(self, valid, p, n, t, prim_id, contrib):
            self.valid, self.p, self.n, self.t, self.prim_id, self.contrib = valid, p, n, t, prim_id, contrib

    class ClosestPointRecord3D:
        def __init__(self, valid, p, n, uv, prim_id, contrib):
            self.valid, self.p, self.n, self.uv, self.prim_id, self.contrib = valid, p, n, uv, prim_id, contrib

    class _Scene:
        dim = 2

        def __init__(self, vertices, indices, values, use_bvh=False, source_type=0, source_params=None):
            self.vertices, self.indices, self.values = vertices, indices, values
            self.use_bvh = use_bvh
            self.source_type, self.source_params = source_type, source_params
            V = vertices.numpy().astype(np.float32)
            F = indices.numpy().astype(np.int64)
            self.normals = (D.Array2 if self.dim == 2 else D.Array3)(_vertex_normals(V, F))
            # bounding box (include/scene.cuh:428-435)
            self.aabb_min, self.aabb_max = V.min(0), V.max(0)

        def largest_inscribed_ball(self, its, epsilon=1e-3):
            """include/scene.cuh:225-249: 10 bisection steps on [epsilon,
            min extent / 2] of the ball tangent at its.p along its.n,
            accepting a radius m when |sdf(p + n m) - m| < 1e-5 (a float
            compared with the double literal)."""
            w = D.width(its.p)
            b0 = np.float32((self.aabb_max - self.aabb_min).min() / np.float32(2))
            a = np.full(w, np.float32(epsilon), np.float32)
            b = np.full(w, b0, np.float32)
            for _ in range(10):
                m = ((a + b) / np.float32(2)).astype(np.float32)
                q = its.p + its.n * D.Float(m)
                with D.suspend_grad():
                    d = np.abs(self.sdf(q).v).astype(np.float32)
                acc = np.abs(d - m).astype(np.float64) < 1e-5
                a = np.where(acc, m, a)
                b = np.where(acc, b, m)
            valid = np.broadcast_to(its.valid.v, (w,))
            return D.Float(np.where(valid, a, np.float32(0)))

    class Scene(_Scene):
        dim = 2

    class Scene3D(_Scene):
        dim = 3

    class _NoWalk:
        def __init__(self, *a, **k):
            pass

        def single_walk(self, *a, **k):
            raise NotImplementedError("the reference's CUDA walk (wos_ext) cannot run here")

    m.ClosestPointRecord, m.ClosestPointRecord3D = ClosestPointRecord, ClosestPointRecord3D
    m.Scene, m.Scene3D = Scene, Scene3D
    m.WoS = m.WoS3D = _NoWalk
    return m


def _vertex_normals(V, F):
    """Scene::configure_normal (include/scene.cuh:368-409): 2D sums the two
    unit edge normals (d.y, -d.x) at each vertex, 3D the unit face normals
    weighted by the corner angle atan2(|a x b|, a.b); then normalises."""
    N = np.zeros_like(V, dtype=np.float32)
    if V.shape[1] == 2:
        d = V[F[:, 1]] - V[F[:, 0]]
        n = np.stack([d[:, 1], -d[:, 0]], 1)
        n = n / np.linalg.norm(n, axis=1, keepdims=True)
        for k in range(2):
            np.add.at(N, F[:, k], n)
    else:
        p0, p1, p2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
        n = np.cross(p1 - p0, p2 - p0)
        n = n / np.linalg.norm(n, axis=1, keepdims=True)

        def angle(a, b):
            return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), (a * b).sum(1))

        for k, w in enumerate((angle(p1 - p0, p2 - p0), angle(p2 - p1, p0 - p1), angle(p0 - p2, p1 - p2))):
            np.add.at(N, F[:, k], (w[:, None] * n).astype(np.float32))
    return (N / np.linalg.norm(N, axis=1, keepdims=True)).astype(np.float32)


def load_reference(ref: Path):
    """Import the reference's wos package from `ref` on top of the stand-in.
    Its wos/fwd.py (Dr.Jit/Mitsuba/torch imports) and wos/io.py (image
    libraries, a download at import) are replaced by modules that export the
    same names."""
    for k in [k for k in sys.modules if k == "wos" or k.startswith("wos.") or k in ("wos_ext", "mitsuba")]:
        del sys.modules[k]
    mi = D.make_mitsuba_module()
    sys.modules["mitsuba"] = mi
    sys.modules["wos_ext"] = fake_wos_ext()
    pkg = types.ModuleType("wos")
    pkg.__path__ = [str(ref / "wos")]
    sys.modules["wos"] = pkg
    fwd = types.ModuleType("wos.fwd")
    names = dict(dr=D.make_dr_namespace(), mi=mi, np=np, Float=D.Float, Int=D.Int, Bool=D.Bool, Array2=D.Array2,
                 Array3=D.Array3, Array4=D.Array4, Array2i=D.Array2i, Array3i=D.Array3i, Array4i=D.Array4i,
                 Loop=D.Loop, PCG32=D.PCG32, Tensor=object, Matrix2=object, Quaternion4=object,
                 basedir=ref, EPSILON=1e-3, Path=Path)
    for k, v in names.items():
        setattr(fwd, k, v)
    sys.modules["wos.fwd"] = fwd
    io = types.ModuleType("wos.io")
    io.write_exr = lambda *a, **k: None
    io.read_2d_obj, io.read_3d_obj = reference_obj_readers(ref)
    sys.modules["wos.io"] = io
    mods = types.SimpleNamespace()
    for name in ("utils", "scene", "scene3d", "solver", "wos", "wos3d", "wos_with_source", "wos_grad",
                 "wos_grad_3d", "wos_boundary"):
        setattr(mods, name, importlib.import_module("wos." + name))
    return mods


def reference_obj_readers(ref: Path):
    """read_2d_obj / read_3d_obj from the reference's wos/io.py, executed
    alone: the module itself imports image libraries and downloads a plugin
    at import time, so only these two function definitions are taken from
    its source."""
    src = (ref / "wos" / "io.py").read_text()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ("read_2d_obj", "read_3d_obj")]
    mod = ast.Module(body=keep, type_ignores=[])
    g = {"np": np}
    exec(compile(mod, str(ref / "wos" / "io.py"), "exec"), g)
    return g["read_2d_obj"], g["read_3d_obj"]


# ---------------------------------------------------------------- inputs
def _shapes():
    spec = importlib.util.spec_from_file_location("b200_shapes", REPO / "diff-wos_b200" / "wos" / "shapes.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def star_inputs(n=192):
    S = _shapes()
    V, F = S.star(n)
    g = (np.sin(3 * V[:, 0]) * np.cos(2 * V[:, 1])).astype(np.float32)
    rng = np.random.default_rng(20261204)
    th = rng.uniform(0, 2 * np.pi, 16)
    frac = np.concatenate([rng.uniform(0.05, 0.9, 10), rng.uniform(0.93, 0.985, 6)])
    r = S.star_radius(th) * frac
    P = np.stack([r * np.cos(th), r * np.sin(th)], 1).astype(np.float32)
    # boundary records: the reference's closest points of points just inside
    thb = np.linspace(0.1, 2 * np.pi + 0.1, 16, endpoint=False)
    rb = S.star_radius(thb) * 0.995
    Pb = np.stack([rb * np.cos(thb), rb * np.sin(thb)], 1).astype(np.float32)
    dV = np.stack([np.cos(3 * np.arange(n) * 2 * np.pi / n + 0.4),
                   0.5 + np.sin(2 * np.arange(n) * 2 * np.pi / n)], 1).astype(np.float32)
    return V, F, g, P, Pb, dV


def sphere_inputs(subdiv=1):
    S = _shapes()
    V, F = S.displaced_icosphere(subdiv, 0.15, 3)
    g = S.harmonic_c3(V).astype(np.float32)
    rng = np.random.default_rng(20261205)
    dirs = rng.normal(size=(16, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rf = S.displaced_radius_fn(0.15, 3)
    frac = np.concatenate([rng.uniform(0.05, 0.75, 10), rng.uniform(0.8, 0.85, 6)])
    P = (dirs * (rf(dirs) * frac)[:, None]).astype(np.float32)
    db = rng.normal(size=(16, 3))
    db /= np.linalg.norm(db, axis=1, keepdims=True)
    Pb = (db * (rf(db) * 0.97)[:, None]).astype(np.float32)
    dV = np.stack([np.sin(2 * V[:, 1] + 0.3), np.cos(3 * V[:, 2]), 0.5 + 0.5 * V[:, 0]], 1).astype(np.float32)
    return V, F, g, P, Pb, dV


SOURCE = np.array([2.0, -1.0, 0.3, 1.0, 0.5], np.float32)  # 1.0 sin(2x - y + 0.3) + 0.5


# ---------------------------------------------------------------- estimators
def _stats(x, n, w):
    x = np.asarray(x, np.float64).reshape(n, w)
    return x.mean(1), x.var(1, ddof=1)


def _rep(v, w):
    return np.repeat(np.asarray(v), w, 0)


def _record2(R, its, w):
    return R.scene.ClosestPointRecord(valid=D.Bool(_rep(its.valid.v, w)), p=D.Array2(_rep(its.p.numpy(), w)),
                                      n=D.Array2(_rep(its.n.numpy(), w)), t=D.Float(_rep(its.t.v, w)),
                                      prim_id=D.Int(_rep(its.prim_id.v, w)))


def _record3(R, its, w):
    return R.scene3d.ClosestPointRecord3D(valid=D.Bool(_rep(its.valid.v, w)), p=D.Array3(_rep(its.p.numpy(), w)),
                                          n=D.Array3(_rep(its.n.numpy(), w)), uv=D.Array2(_rep(its.uv.numpy(), w)),
                                          prim_id=D.Int(_rep(its.prim_id.v, w)))


def _save_record(out, key, its, dim):
    out[key + "_valid"] = np.broadcast_to(its.valid.v, (D.width(its.p),)).astype(np.uint8)
    out[key + "_p"] = its.p.numpy().astype(np.float32)
    out[key + "_n"] = its.n.numpy().astype(np.float32)
    out[key + "_tuv"] = (np.stack([its.t.v, np.zeros_like(its.t.v)], 1) if dim == 2 else its.uv.numpy()).astype(
        np.float32)
    out[key + "_prim"] = its.prim_id.v.astype(np.int32)


def _boundary_stats(valid, idx, X, npix, size, w):
    """Per-pixel mean and standard error of WoSBoundary.walk_detector's
    result (wos/wos_boundary.py:13-21: scatter of the per-sample values
    into their pixels, / detector size / nwalks, over npix * w samples)."""
    N = npix * w
    Y = np.zeros((npix, N))
    ok = np.broadcast_to(valid, (N,)) & (idx >= 0) & (idx < npix)
    Y[idx[ok], np.nonzero(ok)[0]] = X[ok]
    scale = npix / size
    return scale * Y.mean(1), scale * Y.std(1, ddof=1) / np.sqrt(N)


def make_estimators(ref: Path, W2=4096, W3=2048, only=None):
    R = load_reference(ref)
    out = {}

    def want(name):
        return only is None or name in only

    def tick(name, t0):
        print(f"  {name}: {time.time() - t0:.1f} s", flush=True)

    # --- 2D star, 192 segments
    V, F, g, P, Pb, dV = star_inputs()
    out.update(s2_V=V, s2_F=F, s2_g=g, s2_P=P, s2_Pb=Pb, s2_dV=dV, s2_source=SOURCE, s2_W=np.int64(W2))
    n = len(P)

    def poly(source=False):
        kw = dict(source_type=2, source_params=D.Float(SOURCE)) if source else {}
        return R.scene.Polyline(D.Array2(V), D.Array2i(F), D.Float(g), **kw)

    scene = poly()
    prep = D.Array2(_rep(P, W2))
    if want("walk2"):
        t0 = time.time()
        s = R.wos.WoS(nwalks=W2, nsteps=64, epsilon=1e-3)
        v = s.single_walk(prep, scene, D.PCG32(size=n * W2, initstate=11))
        out["walk2_mean"], out["walk2_var"] = _stats(v.v, n, W2)
        tick("walk2", t0)
    if want("walk2_src"):
        scene_s = poly(True)
        for is_ in (False, True):
            t0 = time.time()
            key = "walk2_src_is" if is_ else "walk2_src"
            s = R.wos_with_source.WoSWithSource(nwalks=W2, nsteps=64, epsilon=1e-3, use_IS_for_greens=is_)
            v = s.single_walk(prep, scene_s, D.PCG32(size=n * W2, initstate=12 + is_))
            out[key + "_mean"], out[key + "_var"] = _stats(v.v, n, W2)
            tick(key, t0)
    its = scene.closest_point(D.Array2(Pb))
    _save_record(out, "rec2", its, 2)
    nb = len(Pb)
    if want("tangent2"):
        tx, ty = scene.tangent_derivative(its)
        out["tangent2"] = np.stack([tx.v, ty.v], 1)
        tx, ty = R.wos.WoS().tangent_derivative(its, scene, None)
        out["tangent2_wos"] = np.stack([tx.v, ty.v], 1)
    if want("nd2"):
        t0 = time.time()
        out["nd2_R"] = scene.largest_inscribed_ball(its.c_object()).v
        s = R.wos.WoS(nwalks=W2, nsteps=64, epsilon=1e-3)
        gx, gy = s.normal_derivative(_record2(R, its, W2), scene, D.PCG32(size=nb * W2, initstate=14), clamping=0.1)
        mx, vx = _stats(gx.v, nb, W2)
        my, vy = _stats(gy.v, nb, W2)
        out["nd2_mean"], out["nd2_var"] = np.stack([mx, my], 1), np.stack([vx, vy], 1)
        tick("nd2", t0)
    if want("nd2_src"):
        t0 = time.time()
        scene_s = poly(True)
        its_s = scene_s.closest_point(D.Array2(Pb))
        s = R.wos_with_source.WoSWithSource(nwalks=W2, nsteps=64, epsilon=1e-3)
        gx, gy = s.normal_derivative(_record2(R, its_s, W2), scene_s, D.PCG32(size=nb * W2, initstate=15),
                                     clamping=0.1)
        mx, vx = _stats(gx.v, nb, W2)
        my, vy = _stats(gy.v, nb, W2)
        out["nd2_src_mean"], out["nd2_src_var"] = np.stack([mx, my], 1), np.stack([vx, vy], 1)
        tick("nd2_src", t0)
    if want("ours2"):
        t0 = time.time()
        sc = poly()
        D.set_grad(sc.vertices, D.Array2(dV))
        s = R.wos_grad.Ours(nwalks=W2, nsteps=64, epsilon=1e-3)
        res = s.single_walk(prep, sc, D.PCG32(size=n * W2, initstate=16))
        assert np.all(res.v == 0)
        out["ours2_mean"], out["ours2_var"] = _stats(D.grad(res).v, n, W2)
        tick("ours2", t0)
    if want("boundary2"):
        t0 = time.time()
        sc = poly()
        D.set_grad(sc.vertices, D.Array2(dV))
        det = R.scene.Detector(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(8, 8))
        wb = R.wos_boundary.WoSBoundary(nwalks=W2)
        npix = 64
        valid, idx, val = wb.sample_boundary(sc, det, D.PCG32(size=npix * W2, initstate=17))
        size = float(det.size().v[0])
        out["boundary2_mean"], out["boundary2_se"] = _boundary_stats(valid.v, idx.v, D.grad(val).v, npix, size, W2)
        tick("boundary2", t0)

    # --- 3D displaced icosphere, 80 triangles
    V, F, g, P, Pb, dV = sphere_inputs()
    out.update(s3_V=V, s3_F=F, s3_g=g, s3_P=P, s3_Pb=Pb, s3_dV=dV, s3_W=np.int64(W3))
    n = len(P)

    def mesh():
        return R.scene3d.Scene3D(D.Array3(V), D.Array3i(F), D.Float(g))

    scene = mesh()
    prep = D.Array3(_rep(P, W3))
    if want("walk3"):
        t0 = time.time()
        s = R.wos3d.WoS3D(nwalks=W3, nsteps=128, epsilon=1e-3)
        v = s.single_walk(prep, scene, D.PCG32(size=n * W3, initstate=21))
        out["walk3_mean"], out["walk3_var"] = _stats(v.v, n, W3)
        tick("walk3", t0)
    its = scene.closest_point(D.Array3(Pb))
    _save_record(out, "rec3", its, 3)
    nb = len(Pb)
    if want("tangent3"):
        t = R.wos3d.WoS3D().tangent_derivative(its, scene)
        out["tangent3"] = np.stack([c.v for c in t], 1)
    if want("nd3"):
        t0 = time.time()
        out["nd3_R"] = scene.largest_inscribed_ball(its.c_object()).v
        s = R.wos3d.WoS3D(nwalks=W3, nsteps=128, epsilon=1e-3)
        gr = s.normal_derivative(_record3(R, its, W3), scene, D.PCG32(size=nb * W3, initstate=22), clamping=0.1)
        st = [_stats(c.v, nb, W3) for c in gr]
        out["nd3_mean"], out["nd3_var"] = np.stack([m for m, _ in st], 1), np.stack([v for _, v in st], 1)
        tick("nd3", t0)
    if want("ours3"):
        t0 = time.time()
        sc = mesh()
        D.set_grad(sc.vertices, D.Array3(dV))
        s = R.wos_grad_3d.Ours3D(nwalks=W3, nsteps=128, epsilon=1e-3, epsilon2=1e-3, clamping=0.1)
        # Ours3D walks with the C++ WoS3DCUDA (wos/wos_grad_3d.py:110-115);
        # the reference's own Python WoS3D (wos/wos3d.py:34-61) stands in
        s.wos = R.wos3d.WoS3D(nwalks=W3, nsteps=128, epsilon=1e-3)
        s.wos2 = R.wos3d.WoS3D(nwalks=W3, nsteps=128, epsilon=1e-3)
        res = s.single_walk(prep, sc, D.PCG32(size=n * W3, initstate=23))
        out["ours3_mean"], out["ours3_var"] = _stats(D.grad(res).v, n, W3)
        tick("ours3", t0)
    if want("boundary3"):
        t0 = time.time()
        sc = mesh()
        D.set_grad(sc.vertices, D.Array3(dV))
        det = R.scene3d.Detector3D(vmin=(-1.0, -1.0), vmax=(1.0, 1.0), res=(8, 8), z=D.Float(0.05))
        wb = R.wos_boundary.WoSBoundary(nwalks=W3)
        npix = 64
        valid, idx, val = wb.sample_boundary(sc, det, D.PCG32(size=npix * W3, initstate=24))
        size = float(det.size().v[0])
        out["boundary3_mean"], out["boundary3_se"] = _boundary_stats(valid.v, idx.v, D.grad(val).v, npix, size, W3)
        tick("boundary3", t0)
    return out


# ---------------------------------------------------------------- meshes
MESHES_2D = ("wrench", "clover", "teapot")
MESHES_3D = ("bunny", "bunny2")


def make_meshes(ref: Path):
    R = load_reference(ref)
    dst = OUT / "meshes"
    dst.mkdir(exist_ok=True)
    out = {}
    for name in MESHES_2D + MESHES_3D:
        src = ref / "data" / "meshes" / f"{name}.obj"
        shutil.copyfile(src, dst / f"{name}.obj")
        if name in MESHES_2D:
            for flip in (False, True):
                v, i, c = sys.modules["wos.io"].read_2d_obj(str(src), flip_orientation=flip)
                k = f"{name}_flip" if flip else name
                out[k + "_v"], out[k + "_i"], out[k + "_c"] = v, i, c
            pl = R.scene.Polyline.from_obj(str(src), normalize=True)
            out[name + "_norm_v"] = pl.vertices.numpy()
        else:
            v, i, c = sys.modules["wos.io"].read_3d_obj(str(src))
            out[name + "_v"], out[name + "_i"], out[name + "_c"] = v, i, c
    np.savez_compressed(OUT / "meshes_ref.npz", **out)


# ---------------------------------------------------------------- pins of single routines
def make_ericson(ref: Path, n: int = 1500, seed: int = 20241203):
    R = load_reference(ref)
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    B = (A + rng.uniform(-1, 1, (n, 3))).astype(np.float32)
    C = (A + rng.uniform(-1, 1, (n, 3))).astype(np.float32)
    P = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    # points near each Voronoi feature: vertices, edges, face interior
    k = n // 6
    w = rng.dirichlet([1, 1, 1], k).astype(np.float32)
    P[:k] = (w[:, :1] * A[:k] + w[:, 1:2] * B[:k] + w[:, 2:] * C[:k]
             + rng.normal(0, 1e-3, (k, 3))).astype(np.float32)
    P[k:2 * k] = (A[k:2 * k] + rng.normal(0, 1e-2, (k, 3))).astype(np.float32)
    t = rng.uniform(0, 1, (k, 1)).astype(np.float32)
    P[2 * k:3 * k] = (B[2 * k:3 * k] * t + C[2 * k:3 * k] * (1 - t) + rng.normal(0, 1e-2, (k, 3))).astype(np.float32)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pt, uv, d = R.utils.closest_point_triangle(D.Array3(P), D.Array3(A), D.Array3(B), D.Array3(C))
    np.savez_compressed(OUT / "ericson_ref.npz", a=A, b=B, c=C, p=P, pt=pt.numpy(), uv=uv.numpy(),
                        d=np.broadcast_to(d.v, (n,)).astype(np.float32))


def make_g_cdf(ref: Path):
    s = (ref / "include" / "tabulated_G_cdf.cuh").read_text()
    m = re.search(r"G_cdf\[\]\s*=\s*\{(.*?)\}", s, re.S)
    vals = [float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]
    idx = sorted(set(list(range(0, 20)) + list(range(0, len(vals), 97)) + list(range(len(vals) - 20, len(vals)))))
    json.dump({"size": len(vals), "index": idx, "value": [vals[i] for i in idx],
               "source": "include/tabulated_G_cdf.cuh"}, open(OUT / "g_cdf_ref.json", "w"), indent=0)


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("reference", type=Path, help="path of the reference repository (zihay/diff-wos)")
    ap.add_argument("--only", nargs="*", help="g_cdf, ericson, meshes, estimators, or estimator case names")
    a = ap.parse_args()
    ref = a.reference.resolve()
    if not (ref / "wos" / "wos.py").exists():
        ap.error(f"{ref} does not look like the reference repository (no wos/wos.py)")
    parts = set(a.only or ["g_cdf", "ericson", "meshes", "estimators"])
    if "g_cdf" in parts:
        make_g_cdf(ref)
    if "ericson" in parts:
        make_ericson(ref)
    if "meshes" in parts:
        make_meshes(ref)
    cases = parts - {"g_cdf", "ericson", "meshes", "estimators"}
    if "estimators" in parts or cases:
        path = OUT / "ref_estimators.npz"
        old = dict(np.load(path)) if (cases and path.exists()) else {}
        old.update(make_estimators(ref, only=cases or None))
        np.savez_compressed(path, **old)
    print("wrote", sorted(p.name for p in OUT.iterdir() if p.suffix in (".json", ".npz")))
