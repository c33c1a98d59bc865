"""Inputs outside the reference's domain, handled without a fault.

Points with no primitive at a finite distance (NaN, infinite or overflowing
coordinates) end as invalid walks, bit for bit as the oracle has them
(oracle/wos_oracle.cpp, `walk`), in 2D and 3D, beside ordinary points of the
same call; a workspace below the size the library asks for is refused with
WOS_ERR_WORKSPACE before anything is launched, and the next call runs as usual.
None of these cases makes a kernel fault, trap or wait.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import sphere_scene, star_scene

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _bad_points(dim):
    inf, nan = np.inf, np.nan
    rows = [[nan, 0.0, 0.0], [0.0, nan, 0.0], [inf, 0.0, 0.0], [-inf, inf, 0.0], [1e30, 1e30, 0.0],
            [3e38, -3e38, 0.0]]
    if dim == 3:
        rows += [[0.0, 0.0, nan], [0.0, 0.0, -1e30]]
    return np.array(rows, np.float32)[:, :dim]


@pytest.mark.parametrize("dim", [2, 3])
def test_non_finite_points_end_as_invalid_walks(cuda, oracle, dim):
    import wos
    from wos.native import NativeScene, WalkSettings
    V, F, g = star_scene(512) if dim == 2 else sphere_scene(3)
    rng = np.random.default_rng(11)
    good = rng.uniform(-0.3, 0.3, (40, dim)).astype(np.float32)
    bad = _bad_points(dim)
    P = np.ascontiguousarray(np.concatenate([bad, good, bad[::-1]]))
    ns, os_ = NativeScene(V, F, g), oracle.OracleScene(V, F, g)
    wos.device_status(reset=True)
    s = WalkSettings(nwalks=8, nsteps=32, epsilon=1e-3, seed=21)
    vals, steps = ns.values(P, s, want_steps=True)
    prm = oracle.make_params(s.nwalks, s.nsteps, s.epsilon, s.double_sided, s.prevent_fd_artifacts,
                             s.use_IS_for_greens, s.include_source, s.project_unterminated, s.use_bvh,
                             s.walk_offset, s.seed, s.jitter)
    ov, ovalid, osteps = os_.walk_values(P, prm)
    assert np.array_equal(_np(vals), ov)
    assert np.array_equal(_np(steps), osteps)
    nb = len(bad)
    assert not ovalid[:nb].any() and not ovalid[-nb:].any()
    assert ovalid[nb:-nb].any()
    # the per-point solve of the same call: zero means for the invalid points
    mean = _np(ns.solve(P, s))
    assert np.all(mean[:nb] == 0.0) and np.all(mean[-nb:] == 0.0)
    omean, _ = oracle.reduce(ov)
    np.testing.assert_allclose(mean, omean, rtol=1e-12, atol=1e-12)
    assert wos.device_status() == 0


def test_short_workspace_is_refused_and_the_next_call_runs(cuda):
    import torch
    from wos import _lib
    from wos.native import NativeScene, WalkSettings
    V, F, g = star_scene(512)
    ns = NativeScene(V, F, g)
    P = torch.tensor(np.random.default_rng(3).uniform(-0.3, 0.3, (64, 2)).astype(np.float32), device="cuda")
    s = WalkSettings(nwalks=16, nsteps=32, epsilon=1e-3, seed=4)
    c = s.c()
    L = _lib.lib()
    need = L.wos_solve_workspace_size(64, ctypes.byref(c))
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    mean = torch.full((64,), -7.0, dtype=torch.float64, device="cuda")
    var = torch.full((64,), -7.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.wos_solve(ns.h, ctypes.c_void_p(P.data_ptr()), 64, ctypes.byref(c), ctypes.c_void_p(mean.data_ptr()),
                     ctypes.c_void_p(var.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(need - 1),
                     ctypes.c_void_p(stream))
    assert rc == _lib.WOS_ERR_WORKSPACE
    assert b"workspace" in L.wos_last_error_string()
    torch.cuda.synchronize()
    assert np.all(_np(mean) == -7.0)  # nothing was launched
    rc = L.wos_solve(ns.h, ctypes.c_void_p(P.data_ptr()), 64, ctypes.byref(c), ctypes.c_void_p(mean.data_ptr()),
                     ctypes.c_void_p(var.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(need),
                     ctypes.c_void_p(stream))
    assert rc == 0
    assert np.array_equal(_np(mean), _np(ns.solve(P, s)))
