"""Generate the golden fixtures in tests/golden/ from the reference sources.

Run in a container where the reference repository is available:

    python tests/golden/make_golden.py /path/to/diff-wos

It writes
  g_cdf_ref.json   entries of the reference's tabulated Green's-function CDF
                   (include/tabulated_G_cdf.cuh), read as text;
  ericson_ref.npz  outputs of the reference's point-triangle routine
                   closest_point_triangle (wos/utils.py:108-173) on seeded
                   inputs, executed on a small numpy stand-in for the Dr.Jit
                   array API (float32, elementwise; Dr.Jit itself is not
                   installable here).
The tests only read these files; nothing at test time touches the reference.
"""
from __future__ import annotations

import importlib.util
import json
import re
import sys
import types
import warnings
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


# ---------------------------------------------------------------- numpy stand-in for Dr.Jit
class Vec:
    def __init__(self, *c):
        if len(c) == 1 and isinstance(c[0], Vec):
            c = c[0].c
        self.c = [np.asarray(x, np.float32) for x in c]

    def _op(self, o, f):
        oc = o.c if isinstance(o, Vec) else [np.float32(o)] * len(self.c)
        return type(self)(*[f(a, b) for a, b in zip(self.c, oc)])

    def __add__(self, o): return self._op(o, lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, lambda a, b: b * a)
    def __getitem__(self, i): return self.c[i]

    @property
    def x(self): return self.c[0]

    @property
    def y(self): return self.c[1]

    @property
    def z(self): return self.c[2]


class Array2(Vec):
    pass


class Array3(Vec):
    pass


def _select(cond, a, b):
    if isinstance(a, Vec) or isinstance(b, Vec):
        n = len(a.c) if isinstance(a, Vec) else len(b.c)
        ac = a.c if isinstance(a, Vec) else [a] * n
        bc = b.c if isinstance(b, Vec) else [b] * n
        T = type(a) if isinstance(a, Vec) else type(b)
        return T(*[np.where(cond, x, y).astype(np.float32) for x, y in zip(ac, bc)])
    return np.where(cond, a, b).astype(np.float32)


def _dot(a, b):
    s = a.c[0] * b.c[0]
    for x, y in zip(a.c[1:], b.c[1:]):
        s = s + x * y
    return s.astype(np.float32)


def _make_fake_dr():
    dr = types.SimpleNamespace()
    dr.select = _select
    dr.dot = _dot
    dr.norm = lambda a: np.sqrt(_dot(a, a)).astype(np.float32)
    dr.inf = np.float32(np.inf)
    return dr


def load_reference_utils(ref: Path):
    fake_wos = types.ModuleType("wos")
    fake_wos.__path__ = []
    fwd = types.ModuleType("wos.fwd")
    fwd.dr = _make_fake_dr()
    fwd.Array2, fwd.Array3 = Array2, Array3
    fwd.Bool = lambda v=True: np.bool_(v)
    fwd.Int = lambda v=0: np.int32(v)
    fwd.Float = lambda v=0.0: np.float32(v)
    fwd.Array2i = Array2
    fwd.np = np
    # names that only appear in annotations of functions not used here
    for name in ("PCG32", "Matrix2", "Transform4f", "Loop", "Tensor"):
        setattr(fwd, name, object)
    fwd.__all__ = ["dr", "Array2", "Array3", "Bool", "Int", "Float", "Array2i", "np", "PCG32", "Matrix2",
                   "Transform4f", "Loop", "Tensor"]
    sys.modules["wos"] = fake_wos
    sys.modules["wos.fwd"] = fwd
    spec = importlib.util.spec_from_file_location("ref_wos_utils", ref / "wos" / "utils.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_ericson(ref: Path, n: int = 1500, seed: int = 20241203):
    utils = load_reference_utils(ref)
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
        pt, uv, d = utils.closest_point_triangle(Array3(*P.T), Array3(*A.T), Array3(*B.T), Array3(*C.T))
    np.savez_compressed(OUT / "ericson_ref.npz", a=A, b=B, c=C, p=P, pt=np.stack(pt.c, 1), uv=np.stack(uv.c, 1),
                        d=np.asarray(d, np.float32))


def make_g_cdf(ref: Path):
    s = (ref / "include" / "tabulated_G_cdf.cuh").read_text()
    m = re.search(r"G_cdf\[\]\s*=\s*\{(.*?)\}", s, re.S)
    vals = [float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]
    idx = sorted(set(list(range(0, 20)) + list(range(0, len(vals), 97)) + list(range(len(vals) - 20, len(vals)))))
    json.dump({"size": len(vals), "index": idx, "value": [vals[i] for i in idx],
               "source": "include/tabulated_G_cdf.cuh"}, open(OUT / "g_cdf_ref.json", "w"), indent=0)


if __name__ == "__main__":
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    make_g_cdf(ref)
    make_ericson(ref)
    print("wrote", sorted(p.name for p in OUT.iterdir() if p.suffix in (".json", ".npz")))
