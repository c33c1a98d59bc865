"""Host-side pieces of bench.py that need no GPU: the steps-per-walk
statistics, the gradient-check report and the oracle CPU baselines of the 3D
and batched workloads, on small inputs."""
from __future__ import annotations

import importlib.util
import sys
import types
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_walk_steps_histogram(bench):
    import torch
    steps = torch.tensor([[1, 4, 5, 8], [9, 16, 17, 31], [32, 32, 2, 3]], dtype=torch.int32)
    s = bench.walk_steps(steps, 32)
    assert s["walks"] == 12
    assert abs(sum(s["histogram"].values()) - 1.0) < 1e-12
    assert s["histogram"] == {"0-4": 4 / 12, "5-8": 2 / 12, "9-16": 2 / 12, "17-31": 2 / 12, ">=32": 2 / 12}
    assert s["truncated_fraction"] == 2 / 12
    assert list(bench.walk_steps(steps, 64)["histogram"]) == ["0-4", "5-8", "9-16", "17-32", "33-63", ">=64"]


def test_fd_line_reports_the_configured_step(bench):
    res = {"vertices": [1, 2], "adjoint_mean": [0.0, 1.0],
           "checks": {"h0.001": {"within_2se": 0.5}, "h0.0005": {"within_2se": 1.0}}}
    line = bench.fd_line("w", 10, 4, 2.0, res, "note", (1e-3, 5e-4), 1e-3)
    assert line["value"] == 0.5 and line["ms_per_step"] == 500.0
    assert line["checks"]["h0.0005"]["within_2se"] == 1.0
    assert line["config"]["h"] == [1e-3, 5e-4] and line["config"]["epsilon"] == 1e-3
    # the headline value is the first step asked for
    assert bench.fd_line("w", 10, 4, 2.0, res, "note", (5e-4, 1e-3), 1e-2)["value"] == 1.0


def test_c3_cpu_baseline_small(bench, oracle):
    from wos import shapes
    V, F = shapes.displaced_icosphere(2, 0.15, seed=0)
    P = shapes.sample_interior_3d(64, shapes.displaced_radius_fn(0.15, 0), seed=1, margin=0.05)
    out = bench.c3_cpu_baseline(V, F, P, 64, 4, target_s=0.05)
    for k in ("cpu_baseline", "cpu_baseline_brute_forward"):
        assert out[k]["value"] > 0 and out[k]["kind"] == "port" and out[k]["unit"] == "walks/s"


def test_batched_cpu_baseline_small(bench, oracle):
    import torch
    from wos import shapes
    scenes = shapes.batched_scenes(seed=0, n_stars=2, n_spheres=2, scale=0.01, sphere_levels=(2,))
    items, exact = [], []
    for sc in scenes:
        c = sc["V"].mean(0)
        P = (c + 0.3 * (sc["V"][:4] - c)).astype(np.float32)
        items.append(types.SimpleNamespace(points=torch.as_tensor(P)))
        exact.append(shapes.harmonic_poly(P, sc["coeffs"], sc["degree"]))
    out = bench.batched_cpu_baseline(scenes, items, exact, every=1, m=2)
    assert out["value"] > 0 and out["unit"] == "points/s"


def test_other_workloads_report_each_entry_and_survive_a_failure(bench, monkeypatch):
    """The 3D and batched entries of the default line run at their configured
    sizes with their own step counts, and a failing entry is reported as an
    error without losing the other one (the 2D line is printed either way)."""
    import argparse
    seen = {}

    def fake_c3(ns, compact=False):
        seen["c3"] = (ns.points, ns.walks, ns.steps, ns.warmup, compact)
        return {"value": 1.0}

    def fake_batched(ns, compact=False):
        seen["batched"] = (ns.scale, ns.steps, ns.warmup, compact)
        raise RuntimeError("no memory")

    monkeypatch.setattr(bench, "c3_line", fake_c3)
    monkeypatch.setattr(bench, "batched_line", fake_batched)
    args = argparse.Namespace(steps=20, warmup=5, points=7, walks=None, scale=0.1, no_cpu_baseline=False)
    out = bench.other_workloads(args)
    assert seen["c3"] == (1_000_000, 128, 2, 3, True)
    assert seen["batched"] == (1.0, 1, 1, True)
    assert out["c3_3d_forward_adjoint"]["value"] == 1.0
    assert out["c5_batched"]["error"] == "RuntimeError: no memory"
    assert all("wall_s" in v for v in out.values())
