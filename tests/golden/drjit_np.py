"""A numpy stand-in for the part of the Dr.Jit 0.4 / Mitsuba 3 Python API that
the reference's walk-on-spheres estimators use.

Test infrastructure only: tests/golden/make_golden.py loads the reference's own
Python modules (wos/scene.py, wos/wos.py, wos/wos_with_source.py,
wos/wos3d.py, wos/wos_grad.py, wos/wos_grad_3d.py, wos/wos_boundary.py,
wos/solver.py, wos/utils.py) on top of this module to produce golden
statistics; the product never imports it.  Dr.Jit and Mitsuba themselves are
not installable here.

Semantics (those of Dr.Jit's evaluated "wavefront" mode):
- Float is float32, Float64 float64, Int int32, UInt32 / UInt64 unsigned,
  Bool bool; each array is a 1-D numpy array (width 1 broadcasts).  A Python
  scalar takes the type of the array it meets; mixed array types promote
  (Bool < Int < UInt32 < UInt64 < Float < Float64), as Dr.Jit does.
- Array2 / Array3 (float32) and Array2i / Array3i (int32) hold one array per
  component.
- `Loop(name, state)`: every iteration runs the body on all lanes, then the
  loop-state variables keep their previous values on the lanes whose
  condition was false (Dr.Jit's masked loop).  Other variables assigned in the
  body are updated on every lane, as in the evaluated mode.
- Forward-mode AD: an array may carry a tangent `.t`; arithmetic, sqrt, abs,
  select, min / max, gathers and the vector helpers propagate it, `detach`
  drops it, and `suspend_grad()` stops propagation inside its block.  An
  operation without a derivative rule here raises if a tangent reaches it, so
  no derivative is silently dropped.  `set_grad` seeds a tangent, `grad`
  reads one, `forward_to` is a no-op (tangents are carried eagerly).
- PCG32 is O'Neill's PCG-XSH-RR 64/32 as Dr.Jit implements it: per-lane
  stream inc = ((initseq + lane) << 1) | 1, next_float32 from the top 23
  bits, next_float64 from two 32-bit draws.
- mi.DiscreteDistribution is Mitsuba 3's: CDF accumulated in double and
  stored in float, sampling by binary search for the first CDF entry >= u *
  sum within the range of non-zero entries, and reuse of the sample
  ((u * sum - cdf[i - 1]) / pmf[i]).
"""
from __future__ import annotations

import contextlib
import math
import types

import numpy as np

_GRAD = [True]  # False inside suspend_grad()
# Dr.Jit arithmetic is IEEE without traps: inf / nan results are values
np.seterr(all="ignore")


# ----------------------------------------------------------------- scalar-type arrays
class _Arr:
    dtype = np.float32
    rank = 4
    is_float = True

    def __init__(self, v=0, t=None):
        if isinstance(v, _Arr):
            if t is None and self.is_float and v.is_float:
                t = v.t
            v = v.v
        elif isinstance(v, _Vec):
            raise TypeError("vector given to a scalar-type array")
        v = np.asarray(v)
        if v.dtype == np.bool_ and self.dtype != np.bool_:
            v = v.astype(np.int32)
        if v.ndim == 0:
            v = v.reshape(1)
        if v.dtype != self.dtype:
            with np.errstate(all="ignore"):
                v = v.astype(self.dtype)
        self.v = v
        self.t = None
        if t is not None and self.is_float and _GRAD[0]:
            self.t = np.broadcast_to(np.asarray(t, self.dtype), self.v.shape) if np.ndim(t) else \
                np.full(self.v.shape, t, self.dtype)

    def __len__(self):
        return self.v.shape[0]

    def numpy(self):
        return self.v.copy()

    def __repr__(self):
        return f"{type(self).__name__}({self.v!r})"

    # arithmetic
    def __add__(self, o): return _bin(self, o, "add")
    def __radd__(self, o): return _bin(o, self, "add")
    def __sub__(self, o): return _bin(self, o, "sub")
    def __rsub__(self, o): return _bin(o, self, "sub")
    def __mul__(self, o): return _bin(self, o, "mul")
    def __rmul__(self, o): return _bin(o, self, "mul")
    def __truediv__(self, o): return _bin(self, o, "div")
    def __rtruediv__(self, o): return _bin(o, self, "div")
    def __floordiv__(self, o): return _bin(self, o, "floordiv")
    def __mod__(self, o): return _bin(self, o, "mod")
    def __neg__(self): return _bin(0, self, "sub") if self.is_float else type(self)(-self.v)
    def __pow__(self, o): return power(self, o)
    def __lt__(self, o): return _cmp(self, o, np.less)
    def __le__(self, o): return _cmp(self, o, np.less_equal)
    def __gt__(self, o): return _cmp(self, o, np.greater)
    def __ge__(self, o): return _cmp(self, o, np.greater_equal)
    def __and__(self, o): return _bits(self, o, np.bitwise_and)
    def __rand__(self, o): return _bits(o, self, np.bitwise_and)
    def __or__(self, o): return _bits(self, o, np.bitwise_or)
    def __ror__(self, o): return _bits(o, self, np.bitwise_or)
    def __xor__(self, o): return _bits(self, o, np.bitwise_xor)
    def __rxor__(self, o): return _bits(o, self, np.bitwise_xor)
    def __lshift__(self, o): return type(self)(np.left_shift(self.v, _val(o, self.dtype)))
    def __rshift__(self, o): return type(self)(np.right_shift(self.v, _val(o, self.dtype)))

    def __invert__(self):
        if self.dtype == np.bool_:
            return Bool(~self.v)
        return type(self)(np.invert(self.v))

    # in-place forms mutate this object, so loop-state references stay valid
    def _assign(self, r):
        r = type(self)(r) if not isinstance(r, type(self)) else r
        self.v, self.t = r.v, r.t
        return self

    def __iadd__(self, o): return self._assign(self + o)
    def __isub__(self, o): return self._assign(self - o)
    def __imul__(self, o): return self._assign(self * o)
    def __itruediv__(self, o): return self._assign(self / o)
    def __iand__(self, o): return self._assign(self & o)
    def __ior__(self, o): return self._assign(self | o)

    def __setitem__(self, mask, value):
        m = _mask(mask)
        r = type(self)(value)
        w = max(len(self), len(r), m.shape[0])
        old_v, old_t = _bc(self.v, w), self.t
        self.v = np.where(m, _bc(r.v, w), old_v)
        if self.is_float and (r.t is not None or old_t is not None):
            self.t = np.where(m, _tan(r, w), _tan_of(old_t, w, self.dtype))
        else:
            self.t = None

    def __bool__(self):
        raise TypeError("truth value of an array is ambiguous")

    def __getitem__(self, i):
        # reading one entry gives a Python scalar, as in Dr.Jit
        if isinstance(i, (int, np.integer)):
            return self.v[i].item()
        raise TypeError("array index must be an integer")


class Float(_Arr):
    dtype, rank, is_float = np.float32, 4, True


class Float64(_Arr):
    dtype, rank, is_float = np.float64, 5, True


class Int(_Arr):
    dtype, rank, is_float = np.int32, 1, False


class UInt32(_Arr):
    dtype, rank, is_float = np.uint32, 2, False


class UInt64(_Arr):
    dtype, rank, is_float = np.uint64, 3, False


class Bool(_Arr):
    dtype, rank, is_float = np.bool_, 0, False

    def __init__(self, v=True, t=None):
        super().__init__(v)


_BY_RANK = {0: Bool, 1: Int, 2: UInt32, 3: UInt64, 4: Float, 5: Float64}


def _bc(a, w):
    return a if a.shape[0] == w else np.broadcast_to(a, (w,))


def _val(x, dtype=None):
    if isinstance(x, _Arr):
        return x.v
    return x


def _tan_of(t, w, dtype):
    if t is None:
        return np.zeros(w, dtype)
    return _bc(t, w)


def _tan(a, w):
    return _tan_of(a.t if isinstance(a, _Arr) else None, w, a.dtype if isinstance(a, _Arr) else np.float32)


def _mask(m):
    if isinstance(m, _Arr):
        return m.v.astype(np.bool_)
    return np.asarray(m, np.bool_).reshape(-1)


def _rtype(a, b):
    ra = a.rank if isinstance(a, _Arr) else -1
    rb = b.rank if isinstance(b, _Arr) else -1
    r = max(ra, rb)
    other = b if ra >= rb else a
    if r < 4 and isinstance(other, float):
        r = 4  # an integer array meeting a Python float becomes Float
    return _BY_RANK[r]


def _bin(a, b, op):
    if isinstance(a, _Vec) or isinstance(b, _Vec):
        return _vbin(a, b, op)
    T = _rtype(a, b)
    av = a.v.astype(T.dtype) if isinstance(a, _Arr) and a.dtype != T.dtype else _val(a)
    bv = b.v.astype(T.dtype) if isinstance(b, _Arr) and b.dtype != T.dtype else _val(b)
    with np.errstate(all="ignore"):
        if op == "add":
            r = av + bv
        elif op == "sub":
            r = av - bv
        elif op == "mul":
            r = av * bv
        elif op == "div":
            r = av / bv if T.is_float else np.floor_divide(av, bv)
        elif op == "floordiv":
            r = np.floor_divide(av, bv)
        elif op == "mod":
            r = np.mod(av, bv)
        r = np.asarray(r, T.dtype)
    out = T(r)
    ta = a.t if isinstance(a, _Arr) else None
    tb = b.t if isinstance(b, _Arr) else None
    if T.is_float and _GRAD[0] and (ta is not None or tb is not None):
        w = out.v.shape[0]
        ta = _tan_of(ta, w, T.dtype).astype(T.dtype)
        tb = _tan_of(tb, w, T.dtype).astype(T.dtype)
        A = _bc(np.asarray(av, T.dtype).reshape(-1), w)
        B = _bc(np.asarray(bv, T.dtype).reshape(-1), w)
        with np.errstate(all="ignore"):
            if op == "add":
                t = ta + tb
            elif op == "sub":
                t = ta - tb
            elif op == "mul":
                t = ta * B + A * tb
            elif op == "div":
                t = (ta * B - A * tb) / (B * B)
            else:
                raise NotImplementedError(f"no derivative for {op}")
        out.t = t.astype(T.dtype)
    return out


def _cmp(a, b, f):
    if isinstance(a, _Vec) or isinstance(b, _Vec):
        raise NotImplementedError("vector comparison")
    T = _rtype(a, b)
    av = a.v.astype(T.dtype) if isinstance(a, _Arr) else _val(a)
    bv = b.v.astype(T.dtype) if isinstance(b, _Arr) else _val(b)
    with np.errstate(all="ignore"):
        return Bool(f(av, bv))


def _bits(a, b, f):
    T = _rtype(a, b)
    return T(f(np.asarray(_val(a)).astype(T.dtype), np.asarray(_val(b)).astype(T.dtype)))


# ----------------------------------------------------------------- vectors
class _Vec:
    elem = Float
    n = 2

    def __init__(self, *args):
        E, n = self.elem, self.n
        if len(args) == 0:
            c = [E(0) for _ in range(n)]
        elif len(args) == 1:
            a = args[0]
            if isinstance(a, _Vec):
                c = [E(x) for x in a.c[:n]]
            elif isinstance(a, (tuple, list)) and len(a) == n:
                c = [E(x) for x in a]
            elif isinstance(a, np.ndarray) and a.ndim == 2:
                c = [E(a[:, k]) for k in range(n)]
            else:
                c = [E(a) for _ in range(n)]
        else:
            c = [E(x) for x in args]
        if len(c) != n:
            raise ValueError(f"{type(self).__name__} needs {n} components")
        self.c = c

    def __len__(self):
        return max(len(x) for x in self.c)

    def __repr__(self):
        return f"{type(self).__name__}({[x.v for x in self.c]!r})"

    def numpy(self):
        w = len(self)
        return np.stack([_bc(x.v, w) for x in self.c], 1)

    def __getitem__(self, i):
        if isinstance(i, (int, np.integer)):
            return self.c[i]
        raise TypeError("vector index must be a component number")

    def __setitem__(self, key, value):
        if isinstance(key, (int, np.integer)):
            self.c[key] = self.elem(value)
            return
        vv = value if isinstance(value, _Vec) else type(self)(value)
        for k in range(self.n):
            self.c[k][key] = vv.c[k]

    @property
    def x(self): return self.c[0]

    @x.setter
    def x(self, v): self.c[0] = self.elem(v)

    @property
    def y(self): return self.c[1]

    @y.setter
    def y(self, v): self.c[1] = self.elem(v)

    @property
    def z(self): return self.c[2]

    @z.setter
    def z(self, v): self.c[2] = self.elem(v)

    def __add__(self, o): return _vbin(self, o, "add")
    def __radd__(self, o): return _vbin(o, self, "add")
    def __sub__(self, o): return _vbin(self, o, "sub")
    def __rsub__(self, o): return _vbin(o, self, "sub")
    def __mul__(self, o): return _vbin(self, o, "mul")
    def __rmul__(self, o): return _vbin(o, self, "mul")
    def __truediv__(self, o): return _vbin(self, o, "div")
    def __rtruediv__(self, o): return _vbin(o, self, "div")
    def __neg__(self): return type(self)(*[-x for x in self.c])

    def _assign(self, r):
        self.c = [self.elem(x) for x in r.c]
        return self

    def __iadd__(self, o): return self._assign(self + o)
    def __isub__(self, o): return self._assign(self - o)
    def __imul__(self, o): return self._assign(self * o)
    def __itruediv__(self, o): return self._assign(self / o)


def _vbin(a, b, op):
    V = type(a) if isinstance(a, _Vec) else type(b)
    n = V.n
    ac = a.c if isinstance(a, _Vec) else [a] * n
    bc = b.c if isinstance(b, _Vec) else [b] * n
    r = [_bin(x, y, op) for x, y in zip(ac, bc)]
    if isinstance(a, _Vec) and isinstance(b, _Vec) and type(a) is not type(b):
        V = type(a) if a.elem.rank >= b.elem.rank else type(b)
    return V(*r)


class Array2(_Vec):
    elem, n = Float, 2


class Array3(_Vec):
    elem, n = Float, 3


class Array4(_Vec):
    elem, n = Float, 4


class Array2i(_Vec):
    elem, n = Int, 2


class Array3i(_Vec):
    elem, n = Int, 3


class Array4i(_Vec):
    elem, n = Int, 4


# ----------------------------------------------------------------- loop
def _leaves(objs, out):
    for o in objs:
        if isinstance(o, _Arr):
            out.append(o)
        elif isinstance(o, _Vec):
            out.extend(o.c)
        elif isinstance(o, PCG32):
            out.extend([o.state, o.inc])
        elif isinstance(o, (tuple, list)):
            _leaves(o, out)
        elif hasattr(o, "__dict__"):
            _leaves([v for v in vars(o).values() if isinstance(v, (_Arr, _Vec))], out)
    return out


class Loop:
    """Dr.Jit's masked loop: lanes whose condition is false keep the values
    the loop-state variables had before the body ran."""

    def __init__(self, name="", state=None):
        self.name = name
        self.state = state
        self.mask = None
        self.saved = None

    def __call__(self, cond):
        leaves = _leaves(self.state() if self.state is not None else (), [])
        if self.saved is not None:
            m = self.mask
            w = m.shape[0]
            for leaf, (v, t) in zip(leaves, self.saved):
                ww = max(w, len(leaf))
                leaf.v = np.where(_bc(m, ww), _bc(leaf.v, ww), _bc(v, ww))
                if leaf.is_float and (leaf.t is not None or t is not None):
                    leaf.t = np.where(_bc(m, ww), _tan_of(leaf.t, ww, leaf.dtype), _tan_of(t, ww, leaf.dtype))
        m = _mask(cond)
        if not m.any():
            self.saved = None
            return False
        self.mask = m
        # arrays are never modified in place (every update rebinds .v), so
        # keeping references is a snapshot
        self.saved = None if m.all() else [(leaf.v, leaf.t) for leaf in leaves]
        return True


# ----------------------------------------------------------------- PCG32
_PCG_MULT = np.uint64(0x5851F42D4C957F2D)


class PCG32:
    def __init__(self, size=1, initstate=0x853C49E6748FEA9B, initseq=0xDA3E39CB94B95BDB):
        self.seed(size, initstate, initseq)

    def seed(self, size=1, initstate=0x853C49E6748FEA9B, initseq=0xDA3E39CB94B95BDB):
        lane = np.arange(size, dtype=np.uint64)
        seq = np.asarray(_val(initseq)).astype(np.uint64)
        st0 = np.asarray(_val(initstate)).astype(np.uint64)
        with np.errstate(all="ignore"):
            self.state = UInt64(np.zeros(size, np.uint64))
            self.inc = UInt64(((seq + lane) << np.uint64(1)) | np.uint64(1))
            self.next_uint32()
            self.state = UInt64(self.state.v + st0)
            self.next_uint32()

    def next_uint32(self, mask=True):
        old = self.state.v
        with np.errstate(all="ignore"):
            self.state.v = (old * _PCG_MULT + self.inc.v).astype(np.uint64)
            xs = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
            rot = (old >> np.uint64(59)).astype(np.uint32)
            r = (xs >> rot) | (xs << ((np.uint32(0) - rot) & np.uint32(31)))
        return UInt32(r.astype(np.uint32))

    def next_float32(self, mask=True):
        u = self.next_uint32().v
        return Float(((u >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.0))

    def next_float64(self, mask=True):
        v0 = self.next_uint32().v.astype(np.uint64)
        v1 = self.next_uint32().v.astype(np.uint64)
        u = v0 | (v1 << np.uint64(32))
        return Float64(((u >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0)


# ----------------------------------------------------------------- dr namespace
def _unary(x, f, df=None):
    if isinstance(x, _Vec):
        return type(x)(*[_unary(c, f, df) for c in x.c])
    if not isinstance(x, _Arr):
        x = Float(x) if isinstance(x, float) else Int(x)
    with np.errstate(all="ignore"):
        r = type(x)(np.asarray(f(x.v), x.dtype))
    if x.t is not None and _GRAD[0]:
        if df is None:
            raise NotImplementedError(f"no derivative rule for {f}")
        with np.errstate(all="ignore"):
            r.t = (df(x.v, r.v) * _bc(x.t, len(r))).astype(x.dtype)
    return r


def _to_float(x):
    return x if isinstance(x, (_Arr, _Vec)) else Float(x)


def select(cond, a, b):
    m = _mask(cond)
    if isinstance(a, _Vec) or isinstance(b, _Vec):
        V = type(a) if isinstance(a, _Vec) else type(b)
        ac = a.c if isinstance(a, _Vec) else [a] * V.n
        bc = b.c if isinstance(b, _Vec) else [b] * V.n
        return V(*[select(m, x, y) for x, y in zip(ac, bc)])
    T = _rtype(a, b)
    av = a.v.astype(T.dtype) if isinstance(a, _Arr) else np.asarray(a, T.dtype)
    bv = b.v.astype(T.dtype) if isinstance(b, _Arr) else np.asarray(b, T.dtype)
    out = T(np.where(m, av, bv))
    ta = a.t if isinstance(a, _Arr) else None
    tb = b.t if isinstance(b, _Arr) else None
    if T.is_float and _GRAD[0] and (ta is not None or tb is not None):
        w = len(out)
        out.t = np.where(_bc(m, w), _tan_of(ta, w, T.dtype), _tan_of(tb, w, T.dtype)).astype(T.dtype)
    return out


def dot(a, b):
    s = a.c[0] * b.c[0]
    for x, y in zip(a.c[1:], b.c[1:]):
        s = s + x * y
    return s


def squared_norm(a):
    return dot(a, a)


def norm(a):
    return sqrt(dot(a, a))


def normalize(a):
    return a * rcp(norm(a))


def cross(a, b):
    return Array3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x)


def sqrt(x): return _unary(_to_float(x), np.sqrt, lambda v, r: 0.5 / r)
def abs(x): return _unary(_to_float(x), np.abs, lambda v, r: np.sign(v))  # noqa: A001
def rcp(x): return _unary(_to_float(x), lambda v: 1 / v, lambda v, r: -r * r)
def cos(x): return _unary(_to_float(x), np.cos, lambda v, r: -np.sin(v))
def sin(x): return _unary(_to_float(x), np.sin, lambda v, r: np.cos(v))
def log(x): return _unary(_to_float(x), np.log, lambda v, r: 1 / v)
def exp(x): return _unary(_to_float(x), np.exp, lambda v, r: r)
def acos(x): return _unary(_to_float(x), lambda v: np.arccos(np.clip(v, -1, 1)))
def floor(x): return _unary(_to_float(x), np.floor)
def isfinite(x): return Bool(np.isfinite(_to_float(x).v))


def sign(x):
    x = _to_float(x)
    if isinstance(x, _Vec):
        return type(x)(*[sign(c) for c in x.c])
    return type(x)(np.where(x.v >= 0, 1, -1).astype(x.dtype))


def atan2(y, x):
    y, x = _to_float(y), _to_float(x)
    if y.t is not None or x.t is not None:
        raise NotImplementedError("no derivative rule for atan2")
    return type(y)(np.arctan2(y.v, x.v).astype(y.dtype))


def power(x, p):
    x = _to_float(x)
    return _unary(x, lambda v: np.power(v, x.dtype(p)), lambda v, r: p * np.power(v, x.dtype(p - 1)))


def _componentwise(f, a, b):
    V = type(a) if isinstance(a, _Vec) else type(b)
    ac = a.c if isinstance(a, _Vec) else [a] * V.n
    bc = b.c if isinstance(b, _Vec) else [b] * V.n
    return V(*[f(x, y) for x, y in zip(ac, bc)])


def minimum(a, b):
    if isinstance(a, _Vec) or isinstance(b, _Vec):
        return _componentwise(minimum, a, b)
    return select(_cmp(a, b, np.less_equal), a, b)


def maximum(a, b):
    if isinstance(a, _Vec) or isinstance(b, _Vec):
        return _componentwise(maximum, a, b)
    return select(_cmp(a, b, np.greater_equal), a, b)


def clamp(x, lo, hi):
    return minimum(maximum(x, lo), hi)


def lerp(a, b, t):
    # Dr.Jit: fmadd(b, t, fnmadd(a, t, a)) = a - a t + b t
    return (a - a * t) + b * t


def fmadd(a, b, c):
    return a * b + c


def detach(x):
    if isinstance(x, _Vec):
        return type(x)(*[detach(c) for c in x.c])
    if isinstance(x, _Arr):
        r = type(x)(x.v)
        r.t = None
        return r
    return x


def width(x):
    if isinstance(x, (_Arr, _Vec)):
        return len(x)
    return 1


def gather(T, source, index, active=True):
    idx = _val(index)
    idx = np.asarray(idx).astype(np.int64).reshape(-1)
    m = _mask(active) if not isinstance(active, bool) else None
    if m is not None and m.shape[0] != idx.shape[0]:
        w = max(m.shape[0], idx.shape[0])
        m, idx = _bc(m, w), _bc(idx, w)
    if m is not None:
        idx = np.where(m, idx, 0)

    def g(arr):
        ok = (idx >= 0) & (idx < len(arr))
        v = arr.v[np.clip(idx, 0, len(arr) - 1)]
        v = np.where(ok if m is None else (ok & m), v, np.zeros((), arr.dtype))
        r = type(arr)(v)
        if arr.t is not None and _GRAD[0]:
            tt = _bc(arr.t, len(arr))[np.clip(idx, 0, len(arr) - 1)]
            r.t = np.where(ok if m is None else (ok & m), tt, 0).astype(arr.dtype)
        return r

    if isinstance(source, _Vec):
        return T(*[g(c) for c in source.c])
    return T(g(source))


class ReduceOp:
    Add = "add"


def scatter_reduce(op, target, value, index, active=True):
    if op != ReduceOp.Add:
        raise NotImplementedError(op)
    if isinstance(target, _Vec):
        for k in range(target.n):
            scatter_reduce(op, target.c[k], value.c[k], index, active)
        return
    idx = np.asarray(_val(index)).astype(np.int64).reshape(-1)
    val = _val(value) if isinstance(value, _Arr) else np.asarray(value)
    w = max(idx.shape[0], np.shape(val)[0] if np.ndim(val) else 1)
    idx = _bc(idx, w)
    val = _bc(np.asarray(val, target.dtype).reshape(-1), w)
    m = _bc(_mask(active), w) if not isinstance(active, bool) else np.full(w, active)
    out = target.v.astype(np.float64 if target.is_float else target.dtype).copy()
    np.add.at(out, idx[m], val[m])
    target.v = out.astype(target.dtype)
    if target.is_float and isinstance(value, _Arr) and value.t is not None and _GRAD[0]:
        t = _tan_of(target.t, len(target), target.dtype).astype(np.float64).copy()
        np.add.at(t, idx[m], _bc(value.t, w)[m])
        target.t = t.astype(target.dtype)


def scatter(target, value, index, active=True):
    idx = np.asarray(_val(index)).astype(np.int64).reshape(-1)
    if isinstance(target, _Vec):
        for k in range(target.n):
            scatter(target.c[k], value.c[k], index, active)
        return
    v = target.v.copy()
    v[idx] = _bc(np.asarray(_val(value), target.dtype).reshape(-1), idx.shape[0])
    target.v = v


def arange(T, *a):
    return T(np.arange(*a))


def zeros(T, n=1):
    if issubclass(T, _Vec):
        return T(*[T.elem(np.zeros(n, T.elem.dtype)) for _ in range(T.n)])
    return T(np.zeros(n, T.dtype))


def empty(T, n=1):
    return zeros(T, n)


def full(T, v, n=1):
    if issubclass(T, _Vec):
        return T(*[T.elem(np.full(n, v, T.elem.dtype)) for _ in range(T.n)])
    return T(np.full(n, v, T.dtype))


def linspace(T, start, stop, num, endpoint=True):
    return T(np.linspace(start, stop, num, endpoint=endpoint, dtype=np.float64))


def meshgrid(*arrs, indexing="xy"):
    g = np.meshgrid(*[a.v for a in arrs], indexing=indexing)
    return tuple(type(a)(x.reshape(-1)) for a, x in zip(arrs, g))


def repeat(x, n):
    if isinstance(x, _Vec):
        return type(x)(*[repeat(c, n) for c in x.c])
    r = type(x)(np.repeat(x.v, n))
    if x.t is not None:
        r.t = np.repeat(_bc(x.t, len(x)), n)
    return r


def tile(x, n):
    if isinstance(x, _Vec):
        return type(x)(*[tile(c, n) for c in x.c])
    return type(x)(np.tile(x.v, n))


def prod(x):
    r = x.c[0]
    for c in x.c[1:]:
        r = r * c
    return r


def any(x): return bool(_mask(x).any())  # noqa: A001
def all(x): return bool(_mask(x).all())  # noqa: A001
def none(x): return not bool(_mask(x).any())
def eval(*a): return None  # noqa: A001
def schedule(*a): return None


def sum(x):  # noqa: A001
    return type(x)(np.sum(x.v, dtype=np.float64 if x.is_float else x.dtype))


@contextlib.contextmanager
def suspend_grad(*a, **k):
    old = _GRAD[0]
    _GRAD[0] = False
    try:
        yield
    finally:
        _GRAD[0] = old


@contextlib.contextmanager
def resume_grad(*a, **k):
    old = _GRAD[0]
    _GRAD[0] = True
    try:
        yield
    finally:
        _GRAD[0] = old


def enable_grad(*a):
    return None


def set_grad(x, g):
    if isinstance(x, _Vec):
        gc = g.c if isinstance(g, _Vec) else [g] * x.n
        for c, gg in zip(x.c, gc):
            set_grad(c, gg)
        return
    gv = _val(g)
    x.t = np.broadcast_to(np.asarray(gv, x.dtype).reshape(-1), (len(x),)).copy() if np.ndim(gv) else \
        np.full(len(x), gv, x.dtype)


def grad(x):
    if isinstance(x, _Vec):
        return type(x)(*[grad(c) for c in x.c])
    return type(x)(_tan_of(x.t, len(x), x.dtype))


def forward_to(*a, **k):
    return None


def shape(x):
    return (len(x),) if isinstance(x, _Arr) else (x.n, len(x))


class CustomOp:
    """Base class of dr.custom operations (the reference's _CustomSolver
    subclasses it); custom() evaluates the primal only."""


def custom(cls, *args):
    return cls().eval(*args)


pi = math.pi
inf = float("inf")


def make_dr_namespace():
    ns = types.SimpleNamespace()
    for name in ("select", "dot", "squared_norm", "norm", "normalize", "cross", "sqrt", "abs", "rcp", "cos", "sin",
                 "log", "exp", "acos", "atan2", "floor", "isfinite", "sign", "power", "minimum", "maximum", "clamp",
                 "lerp", "fmadd", "detach", "width", "gather", "scatter_reduce", "scatter", "arange", "zeros",
                 "empty", "full", "linspace", "meshgrid", "repeat", "tile", "prod", "any", "all", "none", "eval",
                 "schedule", "sum", "suspend_grad", "resume_grad", "enable_grad", "set_grad", "grad", "forward_to",
                 "shape"):
        setattr(ns, name, globals()[name])
    ns.ReduceOp = ReduceOp
    ns.CustomOp = CustomOp
    ns.custom = custom
    ns.pi, ns.inf = pi, inf
    ns.Float32, ns.Float64 = Float, Float64
    return ns


# ----------------------------------------------------------------- Mitsuba
class DiscreteDistribution:
    """Mitsuba 3's DiscreteDistribution (sample_reuse_pmf)."""

    def __init__(self, pmf):
        p = np.asarray(_val(pmf), np.float32).reshape(-1)
        cdf = np.cumsum(p.astype(np.float64))
        self.pmf = p
        self.cdf = cdf.astype(np.float32)
        self.sum = np.float32(cdf[-1])
        self.normalization = np.float32(1.0 / cdf[-1])
        nz = np.nonzero(p > 0)[0]
        self.valid = (int(nz[0]), int(nz[-1])) if len(nz) else (0, len(p) - 1)

    def sample_reuse_pmf(self, value):
        u = _to_float(value).v.astype(np.float32) * self.sum
        lo, hi = self.valid
        idx = np.searchsorted(self.cdf, u, side="left")  # first cdf[i] >= u
        idx = np.clip(idx, lo, hi)
        pmf = self.pmf[idx]
        prev = np.where(idx > 0, self.cdf[np.maximum(idx - 1, 0)], np.float32(0))
        with np.errstate(all="ignore"):
            reused = ((u - prev) / pmf).astype(np.float32)
        return Int(idx.astype(np.int32)), Float(reused), Float((pmf * self.normalization).astype(np.float32))

    def eval_pmf_normalized(self, idx):
        return Float(self.pmf[_val(idx)] * self.normalization)


def make_mitsuba_module():
    mi = types.ModuleType("mitsuba")
    mi.DiscreteDistribution = DiscreteDistribution
    mi.set_variant = lambda *a, **k: None

    class _Unavailable:
        def __init__(self, *a, **k):
            raise NotImplementedError("not available in the numpy stand-in")

    mi.Scene = _Unavailable
    mi.Transform4f = _Unavailable
    return mi
