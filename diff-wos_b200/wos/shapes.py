"""Seeded synthetic scenes and query sets (numpy, host side).

These generate the inputs the benchmark configurations are quoted on: the unit
circle polyline, star polylines r(theta) = r0 + a cos(k theta), icospheres with
a radial value-noise displacement, harmonic boundary data and query grids.
Polylines are counter-clockwise and triangle meshes outward-oriented, so the
interior has negative signed distance (include/scene.cuh:155-177).
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------- 2D
def circle(n: int = 1024, radius: float = 1.0, center=(0.0, 0.0)):
    """Closed CCW polyline with n equal segments; vertex k at angle 2 pi k / n."""
    th = 2.0 * np.pi * np.arange(n, dtype=np.float64) / n
    V = np.stack([center[0] + radius * np.cos(th), center[1] + radius * np.sin(th)], 1)
    F = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
    return V.astype(np.float32), F.astype(np.int32)


def star(n: int = 4096, r0: float = 0.6, amp: float = 0.25, lobes: int = 5, phase: float = 0.0):
    """Closed CCW polyline r(theta) = r0 + amp cos(lobes theta + phase), n segments."""
    th = 2.0 * np.pi * np.arange(n, dtype=np.float64) / n
    r = r0 + amp * np.cos(lobes * th + phase)
    V = np.stack([r * np.cos(th), r * np.sin(th)], 1)
    F = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
    return V.astype(np.float32), F.astype(np.int32)


def star_radius(theta, r0=0.6, amp=0.25, lobes=5, phase=0.0):
    return r0 + amp * np.cos(lobes * theta + phase)


def grid(res: int, lo: float = -1.0, hi: float = 1.0):
    """res x res points, x = linspace(lo, hi), y = linspace(hi, lo) (y flipped,
    as Detector.make_points, wos/scene.py:26-31), row-major."""
    x = np.linspace(lo, hi, res, dtype=np.float32)
    y = np.linspace(hi, lo, res, dtype=np.float32)
    X, Y = np.meshgrid(x, y)
    return np.stack([X.ravel(), Y.ravel()], 1).astype(np.float32)


def inside_star(P, r0=0.6, amp=0.25, lobes=5, phase=0.0, margin: float = 0.0):
    th = np.arctan2(P[:, 1], P[:, 0])
    return np.hypot(P[:, 0], P[:, 1]) < star_radius(th, r0, amp, lobes, phase) - margin


# ---------------------------------------------------------------- 3D
def icosphere(subdiv: int = 6):
    """Unit icosphere: 20 * 4^subdiv outward-oriented triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = np.array(V, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(F, np.int64)
    for _ in range(subdiv):
        edges = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.sort(edges, 1)
        uniq, inv = np.unique(key[:, 0] * (len(V) + 1) + key[:, 1], return_inverse=True)
        a = uniq // (len(V) + 1)
        b = uniq % (len(V) + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mid])
        m = inv.reshape(3, -1).T + base  # midpoints of (0,1), (1,2), (2,0)
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([
            np.stack([F[:, 0], m01, m20], 1),
            np.stack([F[:, 1], m12, m01], 1),
            np.stack([F[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1),
        ])
    # orient outward
    c = V[F].mean(1)
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = (n * c).sum(1) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V.astype(np.float32), F.astype(np.int32)


def value_noise3(P, seed: int = 0, octaves: int = 3, base_freq: float = 2.0):
    """Seeded value noise in [-1, 1]: random lattice values, smoothstep
    trilinear interpolation, octaves doubling the frequency, halving amplitude."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)

    def lattice(i, j, k):
        h = perm[(i * 73856093 ^ j * 19349663 ^ k * 83492791) & 4095]
        return table[h]

    out = np.zeros(len(P))
    amp, freq, norm = 1.0, base_freq, 0.0
    for _ in range(octaves):
        X = P * freq
        I = np.floor(X).astype(np.int64)
        f = X - I
        s = f * f * (3 - 2 * f)
        acc = np.zeros(len(P))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) * \
                        (s[:, 2] if dz else 1 - s[:, 2])
                    acc += w * lattice(I[:, 0] + dx, I[:, 1] + dy, I[:, 2] + dz)
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def displaced_icosphere(subdiv: int = 6, amplitude: float = 0.15, seed: int = 0, octaves: int = 3):
    """Icosphere with each vertex moved radially by amplitude * value noise."""
    V, F = icosphere(subdiv)
    V64 = V.astype(np.float64)
    r = 1.0 + amplitude * value_noise3(V64, seed=seed, octaves=octaves)
    return (V64 * r[:, None]).astype(np.float32), F


def displaced_radius_fn(amplitude=0.15, seed=0, octaves=3):
    def f(dirs):
        return 1.0 + amplitude * value_noise3(np.asarray(dirs, np.float64), seed=seed, octaves=octaves)
    return f


def sample_interior_3d(n: int, radius_fn, seed: int = 0, margin: float = 0.0):
    """n uniform points inside a star-shaped surface r(dir) by rejection in its AABB."""
    rng = np.random.default_rng(seed)
    out = []
    got = 0
    while got < n:
        P = rng.uniform(-1.3, 1.3, (max(2 * (n - got), 1024), 3))
        r = np.linalg.norm(P, axis=1)
        ok = r < radius_fn(P / np.maximum(r, 1e-12)[:, None]) - margin
        out.append(P[ok])
        got += int(ok.sum())
    return np.concatenate(out)[:n].astype(np.float32)


# ---------------------------------------------------------------- boundary data
def harmonic_c1(P):
    """x^3 - 3 x y^2 (harmonic)."""
    x, y = P[:, 0].astype(np.float64), P[:, 1].astype(np.float64)
    return x ** 3 - 3 * x * y ** 2


def harmonic_c3(P):
    """x^2 - y^2 + z (harmonic)."""
    x, y, z = (P[:, k].astype(np.float64) for k in range(3))
    return x * x - y * y + z


# ---------------------------------------------------------------- harmonic polynomials
def harmonic_basis(P, degree: int):
    """Harmonic polynomials of degree 1..degree at points P (2D or 3D), one
    column each: Re/Im of (x + iy)^k in 2D; in 3D x, y, z, the degree-2
    harmonics xy, yz, zx, x^2 - y^2, y^2 - z^2 and the degree-3 harmonics
    xyz, x^3 - 3xy^2, y^3 - 3yz^2, z^3 - 3zx^2, x^3 - 3xz^2, y^3 - 3yx^2, z^3 - 3zy^2."""
    P = np.asarray(P, np.float64)
    if P.shape[1] == 2:
        z = P[:, 0] + 1j * P[:, 1]
        cols = []
        for k in range(1, degree + 1):
            w = z ** k
            cols += [w.real, w.imag]
        return np.stack(cols, 1)
    x, y, zz = P[:, 0], P[:, 1], P[:, 2]
    cols = [x, y, zz]
    if degree >= 2:
        cols += [x * y, y * zz, zz * x, x * x - y * y, y * y - zz * zz]
    if degree >= 3:
        cols += [x * y * zz, x ** 3 - 3 * x * y * y, y ** 3 - 3 * y * zz * zz, zz ** 3 - 3 * zz * x * x,
                 x ** 3 - 3 * x * zz * zz, y ** 3 - 3 * y * x * x, zz ** 3 - 3 * zz * y * y]
    return np.stack(cols, 1)


def harmonic_poly(P, coeffs, degree):
    return harmonic_basis(P, degree) @ np.asarray(coeffs, np.float64)


# ---------------------------------------------------------------- batched workload
def batched_scenes(seed: int = 0, n_stars: int = 128, n_spheres: int = 128, scale: float = 1.0,
                   sphere_levels=(3, 4, 5, 6)):
    """Seeded many-scene workload: random star polylines (256-16384 segments,
    3-9 lobes, amplitude 0.1-0.3) and noise-displaced icospheres (1280-81920
    triangles), each with 1k-200k query points (log-uniform, times `scale`)
    and 16-256 walks (log-uniform), boundary data a harmonic polynomial of
    degree 1-3 with coefficients in [-1, 1].  Returns dicts with V, F, g, the
    point count, walks, and the polynomial (degree, coeffs) whose values are
    the exact interior solution.  Query points are drawn by the caller
    (see sample_box) so an exact inside test can filter them."""
    rng = np.random.default_rng(seed)
    base = {}
    out = []
    for i in range(n_stars + n_spheres):
        is_star = i < n_stars
        npts = int(round(np.exp(rng.uniform(np.log(1e3), np.log(2e5))) * scale))
        nwalks = int(round(np.exp(rng.uniform(np.log(16), np.log(256)))))
        deg = int(rng.integers(1, 4))
        if is_star:
            nseg = int(round(np.exp(rng.uniform(np.log(256), np.log(16384)))))
            lobes = int(rng.integers(3, 10))
            amp = float(rng.uniform(0.1, 0.3))
            V, F = star(nseg, 0.6, amp, lobes, phase=float(rng.uniform(0, 2 * np.pi)))
            ncoef = 2 * deg
        else:
            lvl = int(rng.choice(sphere_levels))
            if lvl not in base:
                base[lvl] = icosphere(lvl)
            V0, F = base[lvl]
            V = (V0.astype(np.float64) * (1.0 + 0.15 * value_noise3(V0.astype(np.float64), seed=1000 + i))[:, None])
            V = V.astype(np.float32)
            ncoef = {1: 3, 2: 8, 3: 15}[deg]
        coeffs = rng.uniform(-1, 1, ncoef)
        g = harmonic_poly(V, coeffs, deg).astype(np.float32)
        out.append(dict(V=V, F=F, g=g, dim=V.shape[1], n=max(npts, 1), nwalks=nwalks, degree=deg, coeffs=coeffs,
                        seed=int(rng.integers(0, 2 ** 31))))
    return out


def sample_box(V, n, rng):
    """n uniform points in the bounding box of V."""
    lo, hi = V.min(0), V.max(0)
    return rng.uniform(lo, hi, (n, V.shape[1])).astype(np.float32)
