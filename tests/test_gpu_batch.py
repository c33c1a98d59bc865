"""The batched multi-scene launch against per-item single-scene calls.

Each item's walks are the same Philox walks as in a single-scene call with
the same settings, so per-point means are identical (same reduction order),
and gradients agree up to the order of their FP64 atomic sums.  Graph replay
must give the same results as direct launches, run after run.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _items():
    import torch
    from wos import shapes
    from wos.native import NativeScene as _Native
    from wos.native import WalkSettings
    rng = np.random.default_rng(0)
    items = []

    def NativeScene(V, F, *a):  # noqa: N802 -- keeps the input vertices beside the scene
        ns = _Native(V, F, *a)
        ns.V0 = np.asarray(V, np.float32)
        return ns

    V, F = shapes.circle(512)
    items.append((NativeScene(V, F, shapes.harmonic_c1(V).astype(np.float32)),
                  rng.uniform(-0.6, 0.6, (700, 2)), WalkSettings(nwalks=32, nsteps=64, seed=1), 1))
    V, F = shapes.star(1024, 0.6, 0.2, 4)
    items.append((NativeScene(V, F, np.cos(3 * V[:, 0]).astype(np.float32), 2, [1.0, 2.0, 0.3, 0.5, 1.0]),
                  rng.uniform(-0.3, 0.3, (500, 2)),
                  WalkSettings(nwalks=16, nsteps=64, seed=2, include_source=True, use_IS_for_greens=True), 2))
    V, F = shapes.displaced_icosphere(3, 0.15, 3)
    items.append((NativeScene(V, F, shapes.harmonic_c3(V).astype(np.float32)),
                  rng.uniform(-0.5, 0.5, (400, 3)), WalkSettings(nwalks=24, nsteps=64, seed=3), 1))
    V, F = shapes.star(2048, 0.6, 0.25, 7)
    items.append((NativeScene(V, F, np.sin(2 * V[:, 1]).astype(np.float32)),
                  rng.uniform(-0.3, 0.3, (900, 2)), WalkSettings(nwalks=8, nsteps=32, seed=4), 0))
    out = []
    for sc, P, s, kind in items:
        P = torch.tensor(P.astype(np.float32), device="cuda")
        tg = None
        if kind == 2:
            tg = torch.tensor(rng.normal(size=len(P)).astype(np.float32), device="cuda")
        if kind == 0:
            tg = torch.tensor(rng.normal(size=len(P)).astype(np.float32) * 1e-3, device="cuda")
        out.append((sc, P, s, kind, tg))
    return out


def _np(t):
    return t.detach().cpu().numpy()


def test_batch_matches_single_scene_calls(cuda):
    from wos import BatchItem, BatchPlan
    from wos.native import AdjointSettings
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=True)
    items = _items()
    plan = BatchPlan([BatchItem(sc, P, s, kind, tg) for sc, P, s, kind, tg in items], a)
    info = plan.info()
    assert info["groups"] == 2
    assert info["walks"] == sum(len(P) * s.nwalks for _, P, s, _, _ in items)
    for use_graph in (False, True, True):
        plan.run(use_graph=use_graph)
        for i, (sc, P, s, kind, tg) in enumerate(items):
            o = plan.outputs(i)
            r = sc.solve_adjoint(P, s, a, loss_kind=kind, target=tg, want_var=True)
            assert np.array_equal(_np(o["mean"]), _np(r["mean"])), i
            assert np.array_equal(_np(o["var"]), _np(r["var"])), i
            if kind != 0:
                np.testing.assert_allclose(_np(o["loss"]), _np(r["loss"]), rtol=1e-12)
            for k in ("dV", "dg", "dsrc"):
                x, y = _np(o[k]), _np(r[k])
                np.testing.assert_allclose(x, y, rtol=1e-4, atol=1e-6 * max(np.abs(y).max(), 1e-12)), (i, k)
    import wos
    assert wos.device_status() == 0
    plan.close()


def test_batch_forward_only(cuda):
    from wos import BatchItem, BatchPlan
    items = _items()
    plan = BatchPlan([BatchItem(sc, P, s, kind, tg) for sc, P, s, kind, tg in items], None)
    plan.run(use_graph=True)
    for i, (sc, P, s, kind, tg) in enumerate(items):
        o = plan.outputs(i)
        assert o["dV"] is None
        assert np.array_equal(_np(o["mean"]), _np(sc.solve(P, s)))
    plan.close()


def _batched_items(n_stars, n_spheres, scale, seed=0):
    import torch
    from wos import BatchItem, shapes
    from wos.native import NativeScene, WalkSettings
    rng = np.random.default_rng(seed + 1)
    items, exact = [], []
    for sc in shapes.batched_scenes(seed=seed, n_stars=n_stars, n_spheres=n_spheres, scale=scale,
                                    sphere_levels=(3, 4)):
        ns = NativeScene(sc["V"], sc["F"], sc["g"])
        parts, got = [], 0
        while got < sc["n"]:
            cand = shapes.sample_box(sc["V"], 4096, rng)
            ins = ns.closest(cand, True, want=("inside",))["inside"].bool()
            parts.append(torch.as_tensor(cand, device="cuda")[ins])
            got += int(ins.sum())
        P = torch.cat(parts)[:sc["n"]].contiguous()
        ex = shapes.harmonic_poly(P.cpu().numpy(), sc["coeffs"], sc["degree"])
        s = WalkSettings(nwalks=sc["nwalks"], nsteps=128, epsilon=1e-3, seed=sc["seed"])
        items.append(BatchItem(ns, P, s, 2, torch.as_tensor(ex.astype(np.float32), device="cuda")))
        exact.append(ex)
    return items, exact


def test_batched_harmonic_scenes_match_exact_solution(cuda):
    """Seeded many-scene workload: every scene's field RMSE against the
    exact harmonic polynomial is at the Monte Carlo standard error."""
    from wos import BatchPlan
    from wos.native import AdjointSettings
    items, exact = _batched_items(6, 4, 0.02)
    plan = BatchPlan(items, AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True))
    plan.run(use_graph=True)
    for i, it in enumerate(items):
        o = plan.outputs(i)
        m, v = _np(o["mean"]), _np(o["var"])
        rmse = np.sqrt(((m - exact[i]) ** 2).mean())
        rse = np.sqrt((v / it.settings.nwalks).mean())
        assert rmse < 1.2 * rse + 5e-3, (i, rmse, rse)
        assert np.isfinite(_np(o["dV"])).all() and np.isfinite(_np(o["dg"])).all()
    plan.close()


def test_autotuned_launch_shape_does_not_change_results(cuda):
    """Walks are defined by their Philox counters, so the launch shape the
    tuner picks changes speed only: means are bit-identical."""
    from wos import BatchPlan, autotune
    items, _ = _batched_items(3, 2, 0.01, seed=7)
    plan = BatchPlan(items, None)
    plan.run(use_graph=False)
    ref = [_np(plan.outputs(i)["mean"]) for i in range(len(items))]
    best, times = autotune.tune_batch(plan, candidates=[(128, 16), (512, 64)], repeats=1)
    assert best in times and len(times) == 2
    for bt, chunk in ((128, 16), (512, 64), best):
        plan.set_launch(bt, 0, chunk)
        plan.run(use_graph=True)
        for i in range(len(items)):
            assert np.array_equal(_np(plan.outputs(i)["mean"]), ref[i]), (bt, chunk, i)
    plan.close()


def test_slot_tuner_picks_shapes_per_dimension_and_phase(cuda):
    """wos_batch_autotune_slots keeps one launch shape per (dimension, phase)
    slot present in the plan; results stay bit-identical whatever it picks
    (also when it timed only a prefix of each run's walks)."""
    from wos import BatchPlan, autotune
    from wos.native import AdjointSettings
    items, _ = _batched_items(3, 2, 0.01, seed=8)
    adj = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=False)
    plan = BatchPlan(items, adj)
    plan.run(use_graph=False)
    ref = [(_np(plan.outputs(i)["mean"]), _np(plan.outputs(i)["dg"])) for i in range(len(items))]
    cands = [(128, 0, 16), (256, 2, 32), (512, 0, 64)]
    chosen, times = autotune.tune_batch_slots(plan, candidates=cands, repeats=1, sample=0.5)
    assert set(chosen) == {(2, 0), (2, 1), (3, 0), (3, 1)}
    for slot, c in chosen.items():
        assert c in cands and plan.launch(*slot) == c
        assert len(times[slot]) == 3 and all(np.isfinite(v) and v > 0 for v in times[slot].values())
    plan.run(use_graph=True)
    for i in range(len(items)):
        m, dg = ref[i]
        assert np.array_equal(_np(plan.outputs(i)["mean"]), m), i
        np.testing.assert_allclose(_np(plan.outputs(i)["dg"]), dg, rtol=1e-5, atol=1e-7 * np.abs(dg).max())
    plan.close()


def test_plan_follows_scene_updates_without_refresh(cuda):
    """A plan keeps the scenes it was built from: after their vertices move
    (wos_scene_update_vertices rebuilds the trees in their buffers) or their
    source changes, the next run -- graph replay included, no explicit
    refresh -- equals single-scene calls on the changed scenes."""
    import torch
    from wos import BatchItem, BatchPlan
    from wos.native import AdjointSettings
    a = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=True)
    items = _items()
    plan = BatchPlan([BatchItem(sc, P, s, kind, tg) for sc, P, s, kind, tg in items], a)
    plan.run(use_graph=True)
    before = _np(plan.outputs(0)["mean"]).copy()
    for i, f in ((0, 1.1), (2, 1.05), (3, 1.08)):
        sc = items[i][0]
        sc.update_vertices(torch.as_tensor(sc.V0 * f, device="cuda"))
    items[1][0].set_source(2, [0.5, -1.0, 0.2, 0.3, 2.0])
    for _ in range(2):
        plan.run(use_graph=True)
        for i, (sc, P, s, kind, tg) in enumerate(items):
            o = plan.outputs(i)
            r = sc.solve_adjoint(P, s, a, loss_kind=kind, target=tg, want_var=True)
            assert np.array_equal(_np(o["mean"]), _np(r["mean"])), i
            for k in ("dV", "dg", "dsrc"):
                x, y = _np(o[k]), _np(r[k])
                np.testing.assert_allclose(x, y, rtol=1e-4, atol=1e-6 * max(np.abs(y).max(), 1e-12)), (i, k)
    assert not np.array_equal(before, _np(plan.outputs(0)["mean"]))
    import wos
    assert wos.device_status() == 0
    plan.close()
