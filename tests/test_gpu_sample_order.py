"""The adjoint's sample order (wos_set_sample_order) changes speed, not results.

Samples that start from forward records run sorted by boundary primitive
(mode 1, the default) or in (point, walk) order (mode 0).  Each sample draws
from its own Philox counters, so per-point means, per-walk tangents and their
reductions are bit-identical; only the order of the FP64 gradient atomics
differs, which leaves the float gradients equal to ~1e-7 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import sphere_scene, star_scene

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _close(x, y):
    np.testing.assert_allclose(_np(x), _np(y), rtol=1e-6, atol=1e-7 * max(float(np.abs(_np(y)).max()), 1e-12))


def _case(kind):
    import torch
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    rng = np.random.default_rng(5)
    if kind == "star":
        V, F, g = star_scene(1024)
        ns = NativeScene(V, F, g, 2, [1.0, -1.0, 0.3, 0.5, 1.0])
        P = torch.tensor(rng.uniform(-0.4, 0.4, (1500, 2)).astype(np.float32), device="cuda")
        s = WalkSettings(nwalks=32, nsteps=64, seed=3, include_source=True, use_IS_for_greens=True)
        a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=True)
    else:
        V, F, g = sphere_scene(3)
        ns = NativeScene(V, F, g)
        P = torch.tensor(rng.uniform(-0.5, 0.5, (800, 3)).astype(np.float32), device="cuda")
        s = WalkSettings(nwalks=24, nsteps=64, seed=4)
        a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=False)
    return ns, P, s, a


@pytest.mark.parametrize("kind", ["star", "sphere"])
def test_sample_order_leaves_results_unchanged(cuda, kind):
    import wos
    ns, P, s, a = _case(kind)
    out = {}
    try:
        for mode in (0, 1):
            wos.set_sample_order(mode)
            fused = ns.solve_adjoint(P, s, a, loss_kind=1, want_var=True)
            mean, _, rec, dc = ns.solve_records(P, s, want_dcontrib=a.want_dsrc)
            dLdu = (2.0 / len(P)) * mean.float()
            split = ns.adjoint_records(P, s, a, dLdu, rec, dc)
            dV = torch_randn_like(fused["dV"], 1)
            tan = ns.solve_tangent(P, s, a, dV=dV, want_var=True)
            out[mode] = (fused, split, tan)
    finally:
        wos.set_sample_order(1)
    (f0, s0, t0), (f1, s1, t1) = out[0], out[1]
    assert np.array_equal(_np(f0["mean"]), _np(f1["mean"]))
    assert np.array_equal(_np(f0["var"]), _np(f1["var"]))
    for k in ("dV", "dg", "dsrc"):
        if f0[k] is not None:
            _close(f1[k], f0[k])
    for x, y in zip(s1, s0):
        if x is not None:
            _close(x, y)
    for k in ("tangent", "tangent_var"):
        assert np.array_equal(_np(t0[k]), _np(t1[k])), k
    assert wos.device_status() == 0


def torch_randn_like(t, seed):
    import torch
    gen = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn(t.shape, generator=gen, dtype=torch.float32).to(t.device)


def test_batch_sample_order_leaves_results_unchanged(cuda):
    import wos
    from wos import BatchItem, BatchPlan
    items = []
    for kind in ("star", "sphere", "star"):
        ns, P, s, a = _case(kind)
        items.append(BatchItem(ns, P, s, 1, None))
    a = _case("star")[3]
    res = {}
    try:
        for mode in (0, 1):
            wos.set_sample_order(mode)
            plan = BatchPlan(items, a)
            plan.run(use_graph=True)
            res[mode] = [{k: v.clone() if v is not None else None for k, v in plan.outputs(i).items()}
                         for i in range(len(items))]
            plan.close()
    finally:
        wos.set_sample_order(1)
    for o0, o1 in zip(res[0], res[1]):
        assert np.array_equal(_np(o0["mean"]), _np(o1["mean"]))
        for k in ("dV", "dg", "dsrc"):
            if o0.get(k) is not None:
                _close(o1[k], o0[k])
    assert wos.device_status() == 0


def test_records_adjoint_with_minimal_workspace_runs_unsorted(cuda):
    """wos_adjoint_records given only wos_adjoint_workspace_size bytes runs the
    samples in queue order instead of failing, with the same gradients."""
    import ctypes
    import torch
    from wos import _lib
    ns, P, s, a = _case("sphere")
    mean, _, rec, dc = ns.solve_records(P, s)
    dLdu = (2.0 / len(P)) * mean.float()
    ref = ns.adjoint_records(P, s, a, dLdu, rec, dc)
    c, ca = s.c(), a.c()
    small = _lib.lib().wos_adjoint_workspace_size(ns.h)
    full = _lib.lib().wos_adjoint_records_workspace_size(ns.h, len(P), ctypes.byref(c))
    assert full > small
    ws = torch.empty(small, dtype=torch.uint8, device="cuda")
    dV = torch.zeros((ns.nV, 3), dtype=torch.float32, device="cuda")
    dg = torch.zeros(ns.nV, dtype=torch.float32, device="cuda")
    _lib.call("wos_adjoint_records", ns.h, P.data_ptr(), len(P), ctypes.byref(c), ctypes.byref(ca), dLdu.data_ptr(),
              rec.data_ptr(), None, dV.data_ptr(), dg.data_ptr(), None, ws.data_ptr(), small,
              torch.cuda.current_stream().cuda_stream)
    _close(dV, ref[0])
    _close(dg, ref[1])
