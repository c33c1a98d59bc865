"""wos_solve_noalloc, the entry point that allocates no device memory.

It exists for callers that may not allocate on the device (applications that
own the device through their own pool, latency-critical loops, processes
under a device-memory quota).  This file is collected last so that a run
stopping at its first failure has already run every other test.  It checks,
through the C ABI, that two calls in a row give the same per-point means and
variances as wos_solve, that the second call is not disturbed by the first
one's leftovers in the shared scratch array, and that an oversized request
is refused with a clear error.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_noalloc(scene, P, s, mean, var):
    import torch
    from wos import _lib
    c = s.c()
    return _lib.lib().wos_solve_noalloc(scene.h, P.data_ptr(), int(P.shape[0]), ctypes.byref(c), mean.data_ptr(),
                                        var.data_ptr() if var is not None else None,
                                        torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_solve_on_two_calls(cuda):
    import torch
    from wos import _lib, shapes
    from wos.native import NativeScene, WalkSettings
    V, F = shapes.star(2048)
    g = (np.sin(3 * V[:, 0]) * np.cos(2 * V[:, 1])).astype(np.float32)
    scene = NativeScene(V, F, g, 2, [0.0, 0.0, 0.0, 0.0, 1.0])
    rng = np.random.default_rng(3)
    P1 = torch.tensor(rng.uniform(-0.5, 0.5, (4000, 2)).astype(np.float32), device="cuda")
    P2 = torch.tensor(rng.uniform(-0.4, 0.4, (1500, 2)).astype(np.float32), device="cuda")
    calls = [(P1, WalkSettings(nwalks=256, nsteps=64, seed=11, include_source=True, use_IS_for_greens=True)),
             (P2, WalkSettings(nwalks=64, nsteps=32, seed=12, include_source=True))]
    for P, s in calls:  # two calls in a row through the shared scratch array
        mean = torch.full((P.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
        var = torch.full((P.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(_call_noalloc(scene, P, s, mean, var))
        ref_mean, ref_var = scene.solve(P, s, want_var=True)
        np.testing.assert_allclose(mean.cpu().numpy(), ref_mean.cpu().numpy(), rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(var.cpu().numpy(), ref_var.cpu().numpy(), rtol=1e-10, atol=1e-14)
    assert wos_status_clean()


def wos_status_clean():
    import wos
    return wos.device_status() == 0


def test_noalloc_rejects_oversized_request(cuda):
    import torch
    from wos import _lib, shapes
    from wos.native import NativeScene, WalkSettings
    V, F = shapes.circle(64)
    scene = NativeScene(V, F, np.zeros(len(V), np.float32))
    P = torch.zeros((20000, 2), dtype=torch.float32, device="cuda")
    mean = torch.zeros(20000, dtype=torch.float64, device="cuda")
    rc = _call_noalloc(scene, P, WalkSettings(nwalks=256), mean, None)  # 5.12 M walks > 4,194,304
    assert rc == _lib.WOS_ERR_WORKSPACE
    assert b"exceeds the fixed scratch capacity" in _lib.lib().wos_last_error_string()
