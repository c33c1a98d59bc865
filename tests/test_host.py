"""Host-side logic that needs no GPU: synthetic workloads, OBJ I/O, solver
settings (reference semantics of each solver class), the sampler."""
from __future__ import annotations

import numpy as np
import pytest


def test_c1_point_count():
    from wos import shapes
    P = shapes.grid(128, -0.9, 0.9)
    assert len(P[np.hypot(P[:, 0], P[:, 1]) < 1.0]) == 14592


def test_c2_point_count():
    from wos import shapes
    P = shapes.grid(512)
    n = int(shapes.inside_star(P).sum())
    assert abs(n - 80222) < 200


def test_grid_flips_y():
    from wos import shapes
    P = shapes.grid(3)
    assert P[0, 1] == 1.0 and P[-1, 1] == -1.0 and P[0, 0] == -1.0


def test_icosphere_counts_and_orientation():
    from wos import shapes
    V, F = shapes.icosphere(6)
    assert F.shape == (81920, 3) and V.shape == (40962, 3)
    V, F = shapes.displaced_icosphere(3, 0.15, 0)
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    n = np.cross(b - a, c - a)
    assert np.all((n * (a + b + c)).sum(1) > 0)  # outward
    # closed 2-manifold: every edge shared by exactly two faces
    e = np.sort(np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]), 1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    assert np.all(counts == 2)


def test_circle_is_ccw():
    from wos import shapes
    V, F = shapes.circle(64)
    area = 0.5 * np.sum(V[F[:, 0], 0] * V[F[:, 1], 1] - V[F[:, 1], 0] * V[F[:, 0], 1])
    assert area > 0


def test_value_noise_seeded():
    from wos import shapes
    P = np.random.default_rng(0).normal(size=(100, 3))
    a = shapes.value_noise3(P, seed=1)
    assert np.array_equal(a, shapes.value_noise3(P, seed=1))
    assert not np.array_equal(a, shapes.value_noise3(P, seed=2))
    assert np.abs(a).max() <= 1.0


def test_obj_roundtrip(tmp_path):
    from wos import io, shapes
    V, F = shapes.circle(16)
    g = np.arange(16, dtype=np.float32)
    io.write_2d_obj(tmp_path / "c.obj", V, F, g)
    V2, F2, g2 = io.read_2d_obj(tmp_path / "c.obj")
    np.testing.assert_allclose(V2, V, atol=1e-6)
    assert np.array_equal(F2, F) and np.array_equal(g2, g)
    V2, F2, _ = io.read_2d_obj(tmp_path / "c.obj", flip_orientation=True)
    assert np.array_equal(F2, F[:, ::-1])
    T, TF = shapes.icosphere(1)
    io.write_3d_obj(tmp_path / "s.obj", T, TF)
    T2, TF2, g3 = io.read_3d_obj(tmp_path / "s.obj")
    np.testing.assert_allclose(T2, T, atol=1e-6)
    assert np.array_equal(TF2, TF) and len(g3) == 0


class _FakeScene:
    def __init__(self, dim=2, source_type=0, use_bvh=True):
        self.dim = dim
        self.source_type = source_type
        self.use_bvh = use_bvh


def test_solver_semantics_match_reference_classes():
    import wos
    s = _FakeScene(source_type=2)
    # the Dr.Jit WoS projects unterminated walks; the CUDA walk marks them invalid
    assert wos.WoS().walk_settings(s).project_unterminated is True
    assert wos.WoSCUDA().walk_settings(s).project_unterminated is False
    assert wos.WoS3D().walk_settings(_FakeScene(3)).project_unterminated is True
    assert wos.WoS3DCUDA().walk_settings(_FakeScene(3)).project_unterminated is False
    # defaults of the reference dataclasses
    w = wos.WoS()
    assert (w.epsilon, w.nwalks, w.nsteps) == (1e-3, 10, 32)
    base = wos.Solver()
    assert (base.epsilon, base.nwalks, base.nsteps) == (0.005, 20, 4)
    # source term only for the with-source solvers
    assert wos.WoSCUDA().walk_settings(s).include_source is False
    assert wos.WoSWithSourceCUDA().walk_settings(s).include_source is True
    assert wos.WoSWithSourceCUDA().walk_settings(_FakeScene(2, 0)).include_source is False
    assert wos.WoSWithSourceCUDA(use_IS_for_greens=True).walk_settings(s).use_IS_for_greens is True
    # gradients: values from every value solver, source only from the attached (Dr.Jit) variant
    a = wos.WoSWithSource().adjoint_settings(s, True, True, True)
    assert (a.want_dV, a.want_dg, a.want_dsrc) == (False, True, True)
    a = wos.WoSWithSourceCUDA().adjoint_settings(s, True, True, True)
    assert (a.want_dV, a.want_dg, a.want_dsrc) == (False, True, False)
    a = wos.OursCUDA().adjoint_settings(s, True, True, True)
    assert (a.want_dV, a.want_dg, a.want_dsrc) == (True, False, False)
    a = wos.OursCUDA(grad_values=True, grad_source=True, epsilon2=5e-4).adjoint_settings(s, True, True, True)
    assert (a.want_dV, a.want_dg, a.want_dsrc, a.epsilon2) == (True, True, True, 5e-4)
    # the reference's OursCUDA uses the source-blind normal derivative (wos/wos_grad.py:146)
    assert wos.OursCUDA().adjoint_settings(s, True, True, True).source_in_normal_derivative is False
    assert wos.OursCUDA(source_in_normal_derivative=True).adjoint_settings(s, True, False, False) \
        .source_in_normal_derivative is True
    # the reference's Ours: WoS walks (projected at nsteps) at epsilon for the primal and the ball walks
    o = wos.Ours(epsilon=2e-3, epsilon2=7e-4)
    assert o.adjoint_settings(s, True, False, False).epsilon2 == 2e-3
    assert o.walk_settings(s).project_unterminated is True
    assert wos.OursCUDA().walk_settings(s).project_unterminated is False


def test_sampler_advances():
    import wos
    s = wos.Sampler(seed=5, offset=3)
    assert s.take() == 3 and s.take() == 3 + 1 and s.offset == 5
    from wos.solver import as_sampler
    assert as_sampler(9).seed == 9 and as_sampler(s) is s


def test_walk_settings_to_c():
    from wos.native import WalkSettings
    c = WalkSettings(nwalks=7, nsteps=9, epsilon=2e-3, seed=(1 << 63) + 5, walk_offset=(1 << 32) + 3).c()
    assert (c.nwalks, c.nsteps, c.walk_offset, c.seed) == (7, 9, 3, (1 << 63) + 5)


def test_statistics():
    from wos import Statistics
    x = np.random.default_rng(0).normal(size=1000)
    st = Statistics()
    assert np.isclose(st.mean(x)[-1], x.mean())
    assert np.isclose(st.var(x)[-1], x.var())


def test_merge_solves_equals_one_solve_of_all_walks(oracle):
    """A solve resumed over the next walk range: merging the per-point
    (mean, var) of walks [0, a) and [a, a + b) gives the reduction of all
    a + b walks (the oracle's reduction, the GPU k_reduce's restatement)."""
    import torch
    from wos import merge_solves
    rng = np.random.default_rng(5)
    vals = (rng.normal(size=(300, 96)) * rng.uniform(0.1, 3.0, (300, 1)) + 2.0).astype(np.float32)
    for a in (1, 17, 48, 95):
        ma, va = oracle.reduce(np.ascontiguousarray(vals[:, :a]))
        mb, vb = oracle.reduce(np.ascontiguousarray(vals[:, a:]))
        m, v = merge_solves(ma, va, a, mb, vb, 96 - a)
        mall, vall = oracle.reduce(vals)
        np.testing.assert_allclose(m, mall, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(v, vall, rtol=1e-10, atol=1e-12)
        mt, vt = merge_solves(torch.tensor(ma), torch.tensor(va), a, torch.tensor(mb), torch.tensor(vb), 96 - a)
        np.testing.assert_allclose(mt.numpy(), m, rtol=1e-15)
        np.testing.assert_allclose(vt.numpy(), v, rtol=1e-15)
    m, v = merge_solves(np.zeros(3), np.zeros(3), 0, mall[:3], vall[:3], 96)
    assert np.array_equal(m, mall[:3]) and np.array_equal(v, vall[:3])


@pytest.mark.parametrize("dim,degree", [(2, 1), (2, 3), (3, 1), (3, 2), (3, 3)])
def test_harmonic_basis_is_harmonic(dim, degree):
    from wos import shapes
    rng = np.random.default_rng(dim * 10 + degree)
    P = rng.uniform(-1, 1, (64, dim))
    h = 1e-3
    lap = -2 * dim * shapes.harmonic_basis(P, degree)
    for k in range(dim):
        e = np.zeros(dim)
        e[k] = h
        lap = lap + shapes.harmonic_basis(P + e, degree) + shapes.harmonic_basis(P - e, degree)
    assert np.abs(lap / h ** 2).max() < 1e-5
    ncols = shapes.harmonic_basis(P, degree).shape[1]
    assert ncols == (2 * degree if dim == 2 else {1: 3, 2: 8, 3: 15}[degree])


def test_batched_scenes_ranges_and_seeding():
    from wos import shapes
    a = shapes.batched_scenes(seed=5, n_stars=6, n_spheres=3, scale=0.1, sphere_levels=(2, 3))
    b = shapes.batched_scenes(seed=5, n_stars=6, n_spheres=3, scale=0.1, sphere_levels=(2, 3))
    assert len(a) == 9
    for x, y in zip(a, b):
        assert np.array_equal(x["V"], y["V"]) and np.array_equal(x["g"], y["g"]) and x["seed"] == y["seed"]
    for sc in a:
        assert 16 <= sc["nwalks"] <= 256 and 1 <= sc["degree"] <= 3
        assert 100 <= sc["n"] <= 20000
        if sc["dim"] == 2:
            assert 256 <= sc["F"].shape[0] <= 16384
        else:
            assert sc["F"].shape[0] in (320, 1280)
        np.testing.assert_allclose(sc["g"], shapes.harmonic_poly(sc["V"], sc["coeffs"], sc["degree"]), rtol=1e-5,
                                   atol=1e-5)


def test_soft_walk_tangent_formulas_float64():
    """The forward-mode rules of the soft-edge walk (distance motion
    n . (dx - dc) at fixed barycentrics, projection-parameter motion of the
    boundary value, weight and throughput products), restated in float64
    numpy on a brute-force polyline, agree with central differences away
    from the |sdf| kink."""
    from wos import shapes
    V, F = shapes.star(96, 0.6, 0.2, 4)
    V = V.astype(np.float64)
    rng = np.random.default_rng(2)
    g = V[:, 0] ** 2 - V[:, 1] ** 2 + 0.5 * V[:, 0]
    dV = rng.normal(size=V.shape) * 0.2
    dV[:, 0] += 1.0
    dg = rng.normal(size=len(V))
    eps = 5e-2

    def nearest(Vv, x):
        a, b = Vv[F[:, 0]], Vv[F[:, 1]]
        e = b - a
        t = np.clip(((x - a) * e).sum(1) / (e * e).sum(1), 0, 1)
        c = a + t[:, None] * e
        d2 = ((x - c) ** 2).sum(1)
        j = int(np.argmin(d2))
        return j, np.sqrt(d2[j]), t[j], c[j]

    def walk(Vv, gv, x0, dirs, tan=False):
        x, xd = x0.copy(), np.zeros(2)
        beta, betad, res, resd = 1.0, 0.0, 0.0, 0.0
        for om in dirs:
            j, d, t, c = nearest(Vv, x)
            ia, ib = F[j]
            val = gv[ia] + t * (gv[ib] - gv[ia])
            dd = vd = 0.0
            if tan:
                cd = (1 - t) * dV[ia] + t * dV[ib]
                dd = (x - c) / d @ (xd - cd)
                e, ed = Vv[ib] - Vv[ia], dV[ib] - dV[ia]
                td = (((xd - dV[ia]) @ e + (x - Vv[ia]) @ ed) - 2 * t * (e @ ed)) / (e @ e) if 0 < t < 1 else 0.0
                vd = td * (gv[ib] - gv[ia]) + (1 - t) * dg[ia] + t * dg[ib]
            w = min(d, eps) / eps
            wd = dd / eps if d < eps else 0.0
            res += beta * (1 - w) * val
            resd += betad * (1 - w) * val - beta * wd * val + beta * (1 - w) * vd
            betad, beta = betad * w + beta * wd, beta * w
            x, xd = x + d * om, xd + dd * om
        return res, resd

    h = 1e-6
    for k in range(25):
        th = rng.uniform(0, 2 * np.pi, 8)
        dirs = np.stack([np.cos(th), np.sin(th)], 1)
        x0 = rng.uniform(-0.3, 0.3, 2)
        _, tan = walk(V, g, x0, dirs, tan=True)
        fd = (walk(V + h * dV, g + h * dg, x0, dirs)[0] - walk(V - h * dV, g - h * dg, x0, dirs)[0]) / (2 * h)
        assert abs(fd - tan) < 1e-4 * (1 + abs(tan)), (k, fd, tan)
