#!/usr/bin/env python
"""Benchmark of the walk-on-spheres hot path on B200.

Workload (one "step", the 2D differentiable solve): star polyline
r(theta) = 0.6 + 0.25 cos(5 theta) with 4096 CCW segments, Dirichlet data
g = sin(3x) cos(2y) at the vertices, constant source f = 1 (source type 2,
amplitude 0, offset 1) sampled with the tabulated Green's-function CDF,
queries = the 512 x 512 grid on [-1, 1]^2 masked to the interior (80,222
points), 256 walks per point, nsteps 64, epsilon 1e-3.  A step is the
forward solve (per-point means) followed by the adjoint of loss = mean(u^2)
with respect to per-vertex g, the source parameters and the vertex positions
(boundary-shape estimator, epsilon2 1e-3, clamping 0.1).  All inputs are
seeded synthetic data of these shapes.

value   walks/s of whole steps on the device (inputs resident in HBM), summed
        over all ranks; each walk is both a forward walk and an adjoint sample.
e2e     the same metric through the public Python API (wos.CustomSolver with
        WoSWithSourceCUDA forward and OursCUDA backward, torch autograd) with
        host buffers: H2D of points and scene, scene build, forward, backward,
        D2H of loss and gradients inside the timed region.
roofline  the adjoint kernel (the dominant one), which is bound by
        instruction issue: warp instructions per nearest query (from the ncu
        capture in profiles/) x the launch's queries (device counters) / its
        CUDA-event time, against 148 SMs x 4 schedulers x the SM clock.
        Beside it: `ref_lbvh_bytes`, the reference LBVH traversal's box and
        primitive bytes for the same samples over the HBM copy peak (served
        from L1/L2), and `fp32_algorithmic`, the reference algorithm's FP32
        ops (12 per node visit, 20 per segment test, 10 per query) over
        148 SMs x 128 lanes x 2 x SM clock; `traffic` is DRAM bytes.
other_workloads  after the 2D line is complete (one GPU only; skipped with
        --no-other-workloads): the 3D forward + adjoint solve on the displaced
        icosphere at 1,000,000 points x 128 walks, and the 256-scene batch at
        full scale against the plain per-scene kernel, each timed with its own
        CUDA events, clocks, accuracy and CPU baseline (the lines that
        --workload c3 / batched print, without their untimed extras).
--impl reference  the CPU restatement of the reference algorithm (the
        reference itself cannot run: it needs Dr.Jit/Mitsuba and the lbvh
        submodule), all host threads, bounded samples of the same workload.

Multi-GPU (torchrun): every rank runs the same workload with its own seed on
its own GPU (weak scaling, no data-path collective); times are the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "diff-wos_b200"))

import numpy as np  # noqa: E402

METRIC = "wos_walks_per_s"
UNIT = "walks/s"
STAR = dict(n=4096, r0=0.6, amp=0.25, lobes=5)
GRID = 512
NWALKS = 256
NSTEPS = 64
EPS = 1e-3
EPS2 = 1e-3
CLAMP = 0.1
SOURCE = [0.0, 0.0, 0.0, 0.0, 1.0]


# ---------------------------------------------------------------- workload
def set_size(grid, walks):
    global GRID, NWALKS
    GRID, NWALKS = int(grid), int(walks)


def make_workload():
    from wos import shapes
    V, F = shapes.star(STAR["n"], STAR["r0"], STAR["amp"], STAR["lobes"])
    g = (np.sin(3 * V[:, 0]) * np.cos(2 * V[:, 1])).astype(np.float32)
    P = shapes.grid(GRID, -1.0, 1.0)
    P = P[shapes.inside_star(P, STAR["r0"], STAR["amp"], STAR["lobes"])]
    return V, F, g, np.ascontiguousarray(P)


def walk_settings(seed):
    from wos.native import WalkSettings
    return WalkSettings(nwalks=NWALKS, nsteps=NSTEPS, epsilon=EPS, use_IS_for_greens=True, include_source=True,
                        use_bvh=True, seed=seed)


def adjoint_settings():
    from wos.native import AdjointSettings
    return AdjointSettings(epsilon2=EPS2, clamping=CLAMP, control_variates=True, source_in_normal_derivative=True,
                           want_dV=True, want_dg=True, want_dsrc=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        rows = [l.split(", ") for l in self.lines if l]
        if self.uuid:
            mine = [r for r in rows if len(r) > 1 and self.uuid in r[1]]
            rows = mine or rows
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[2]))
                mx.append(float(r[3]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[6:10]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- measured peaks
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(V, F, g, P, target_s=6.0, seed=0):
    """The oracle (C++ restatement of the reference walk, OpenMP, all host
    threads) on a bounded sample of the same step: forward walks + adjoint
    samples at NWALKS walks per point."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    S = O.OracleScene(V, F, g, 2, SOURCE)
    prm = O.make_params(nwalks=NWALKS, nsteps=NSTEPS, epsilon=EPS, use_IS_for_greens=True, include_source=True,
                        use_bvh=True, seed=seed)
    adj = O.make_adj(EPS2, CLAMP, True, True, 1e-3, True, True, True)
    threads = os.cpu_count() or 1

    def run(n):
        idx = np.linspace(0, len(P) - 1, n).astype(np.int64)
        sub = P[idx]
        t0 = time.perf_counter()
        vals, _, _ = S.walk_values(sub, prm, nthreads=threads)
        mean, _ = O.reduce(vals)
        dLdu = (2.0 * mean / len(P)).astype(np.float32)
        S.adjoint(sub, prm, adj, dLdu, nthreads=threads)
        return time.perf_counter() - t0

    probe = 8
    t = run(probe)
    n = int(max(probe, min(len(P), probe * target_s / max(t, 1e-3))))
    return S, prm, adj, run, n, threads


def reference_work(S, prm, adj, P, npts=96):
    """Algorithmic work per walk of the reference algorithm: the oracle's
    deterministic binary LBVH (Karras, leaf size 1, nearest-first, prune when
    the box distance exceeds the best) counts queries, node visits and
    primitive tests for the forward walks and for forward + adjoint samples
    of `npts` points spread over the query set.  Returns per-walk averages
    for the forward walk and for the adjoint part alone."""
    from oracle import oracle as O
    idx = np.linspace(0, len(P) - 1, npts).astype(np.int64)
    sub = P[idx]
    vals, fw = S.walk_counted(sub, prm, nthreads=os.cpu_count() or 1)
    mean, _ = O.reduce(vals)
    dLdu = (2.0 * mean / len(P)).astype(np.float32)
    _, fa = S.adjoint_counted(sub, prm, adj, dLdu, nthreads=os.cpu_count() or 1)
    walks = npts * NWALKS
    fwd = {k: fw[k] / walks for k in fw}
    adjoint = {k: (fa[k] - fw[k]) / walks for k in fa}
    return {"forward": fwd, "adjoint": adjoint, "sample": f"{npts} points x {NWALKS} walks"}


def algorithmic(work, dim=2):
    """Bytes and FP32 ops of the counted work: 16 dim B per node visit (two
    child boxes), 16 B per segment / 36 B per triangle test; 12 / 18 ops per
    node visit, 20 / 60 per primitive test, 10 per query (walk update)."""
    nb, npr, nq = work["nodes"], work["prims"], work["queries"]
    byt = 16.0 * dim * nb + (16.0 if dim == 2 else 36.0) * npr
    ops = (12.0 if dim == 2 else 18.0) * nb + (20.0 if dim == 2 else 60.0) * npr + 10.0 * nq
    return byt, ops


def cpu_info():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    V, F, g, P = make_workload()
    S, prm, adj, run, n, threads = cpu_baseline(V, F, g, P, target_s=args.ref_step_s)
    for _ in range(args.warmup):
        run(n)
    ts = [run(n) for _ in range(args.steps)]
    t = float(np.mean(ts))
    value = n * NWALKS / t
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(len(P)),
        "sample": {"points_per_step": n, "of_points": len(P), "walks_per_point": NWALKS,
                   "note": "each step runs the forward walks and adjoint samples of an evenly spaced subset of the "
                           "workload's points (a bounded CPU sample); walks/s is per walk, so it compares with "
                           "the full-workload GPU figure"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} of {len(P)} points x {NWALKS} walks (forward + adjoint), oracle C++ "
                                   f"restatement, {threads} threads, {cpu_info()}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference needs Dr.Jit/Mitsuba and its lbvh submodule and cannot run; "
                "its algorithm is timed through the C++ restatement",
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(npts):
    c = {"workload": f"2d_differentiable_solve_star4096_grid{GRID}_walks{NWALKS}",
         "scene": "star r=0.6+0.25cos(5t), 4096 segments", "points": npts, "walks_per_point": NWALKS,
         "nsteps": NSTEPS, "epsilon": EPS, "epsilon2": EPS2, "source": "f=1, G-CDF importance sampling",
         "loss": "mean(u^2); adjoint wrt g, f, vertex xy", "nearest": "LBVH",
         "l2": "inputs < L2; 256 MiB buffer written between timed steps (L2 flush)"}
    return c


# ---------------------------------------------------------------- batched workload
def batched_main(args):
    print(json.dumps(batched_line(args)), flush=True)
    return 0


def batched_line(args, compact=False):
    """Many scenes in one plan: persistent launches per dimension and tree depth (graph replay):
    seeded random stars and noise-displaced icospheres, harmonic-polynomial
    boundary data, forward + adjoint of mean((u - exact)^2) per scene.
    Compared with the reference-shaped plain kernel run scene by scene.
    `compact` (the entry in the default bench line): the tuner times 2 % of
    each run's walks, brute force runs on every 8th scene instead of every
    4th, and the per-dimension breakdown plans are left out."""
    import torch
    import wos
    from wos import autotune, shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scenes = shapes.batched_scenes(seed=0, scale=args.scale)
    rng = np.random.default_rng(1)
    items, exact = [], []
    for sc in scenes:
        ns = NativeScene(sc["V"], sc["F"], sc["g"])
        n, parts, got = sc["n"], [], 0
        while got < n:
            cand = shapes.sample_box(sc["V"], max(3 * (n - got), 1024), rng)
            ins = ns.closest(cand, True, want=("inside",))["inside"].bool()
            c = torch.as_tensor(cand, device=dev)[ins]
            parts.append(c)
            got += int(c.shape[0])
        P = torch.cat(parts)[:n].contiguous()
        ex = shapes.harmonic_poly(P.cpu().numpy(), sc["coeffs"], sc["degree"])
        exact.append(ex)
        st = WalkSettings(nwalks=sc["nwalks"], nsteps=64, epsilon=1e-3, seed=sc["seed"])
        items.append(wos.BatchItem(ns, P, st, loss_kind=2,
                                   target=torch.as_tensor(ex.astype(np.float32), device=dev)))
    adj = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=False)
    plan = wos.BatchPlan(items, adj)
    info = plan.info()
    # per (dimension, phase) slot; large plans time a prefix of each run
    sample = min(1.0, (0.02 if compact else 0.1) / max(args.scale, 1e-9))
    slot_best, slot_ms = autotune.tune_batch_slots(plan, sample=sample)
    for _ in range(args.warmup):
        plan.run(use_graph=True)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(None)
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.run(use_graph=True)
        b.record()
        torch.cuda.synchronize()
        t += a.elapsed_time(b) * 1e-3
    clk = clocks.stop()
    ms = t / args.steps * 1e3
    # accuracy of the batched estimates against the exact harmonic solutions
    se2, err2, npts = 0.0, 0.0, 0
    for i, it in enumerate(items):
        o = plan.outputs(i)
        m, v = o["mean"].cpu().numpy(), o["var"].cpu().numpy()
        err2 += float(((m - exact[i]) ** 2).sum())
        se2 += float((v / it.settings.nwalks).sum())
        npts += len(m)
    # the reference-shaped plain kernel (one walk per thread, forward only),
    # scene by scene.  Large scenes run on a subsample of >= 2^18 walks (enough
    # to fill the GPU), scaled by points; small scenes run whole.  Brute force
    # runs on every 4th (compact: 8th) scene and is extrapolated per dimension by its time
    # ratio to the LBVH plain kernel on the same scenes.
    def plain_time(it, use_bvh):
        nw = it.settings.nwalks
        n = it.points.shape[0]
        m = min(n, -(-(1 << 18) // nw))
        s = WalkSettings(nwalks=nw, nsteps=64, epsilon=1e-3, seed=it.settings.seed, use_bvh=use_bvh)
        Ps = it.points[:m]
        it.scene.values(Ps, s, plain=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        it.scene.values(Ps, s, plain=True)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) * 1e-3 * n / m

    t_lbvh = [plain_time(it, True) for it in items]
    t_brute_est = 0.0
    plain_by_dim = {}
    for dim in (2, 3):
        idx = [i for i, it in enumerate(items) if it.scene.dim == dim]
        sub = idx[::8 if compact else 4]
        ratio = sum(plain_time(items[i], False) for i in sub) / sum(t_lbvh[i] for i in sub)
        t_brute_est += ratio * sum(t_lbvh[i] for i in idx)
        npts = sum(items[i].points.shape[0] for i in idx)
        plain_by_dim[f"{dim}d"] = {"lbvh_ms": 1e3 * sum(t_lbvh[i] for i in idx),
                                   "brute_ms": 1e3 * ratio * sum(t_lbvh[i] for i in idx), "points": npts}
    plain = {"lbvh": info["points"] / sum(t_lbvh), "brute": info["points"] / t_brute_est}
    # where the step's time goes: forward-only and forward+adjoint plans per dimension
    def plan_ms(sub, adjoint):
        pl = wos.BatchPlan(sub, adjoint)
        for (d, ph), shape in slot_best.items():
            pl.set_launch_slot(d, ph, *shape)
        pl.run(use_graph=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        pl.run(use_graph=True)
        b.record()
        torch.cuda.synchronize()
        pl.close()
        return a.elapsed_time(b)

    breakdown = {}
    for dim in ((2, 3) if not compact else ()):
        sub = [it for it in items if it.scene.dim == dim]
        breakdown[f"{dim}d"] = {"scenes": len(sub), "walks": sum(it.points.shape[0] * it.settings.nwalks for it in sub),
                                "forward_ms": plan_ms(sub, None), "forward_adjoint_ms": plan_ms(sub, adj)}
    value = info["points"] / (ms * 1e-3)
    line = {
        "metric": "batched_query_points_per_s", "value": value, "unit": "points/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched_{len(items)}_scenes_scale{args.scale:g}", "scenes": len(items),
                   "points": info["points"], "walks": info["walks"], "nsteps": 64, "epsilon": 1e-3,
                   "loss": "sum over scenes of mean((u - exact)^2); adjoint wrt vertices and values",
                   "launch": "one persistent kernel per dimension, tree depth and phase, CUDA graph replay",
                   "l2": "256 MiB buffer written between timed steps (L2 flush)"},
        "walks_per_s": info["walks"] / (ms * 1e-3),
        "autotuned_launch": {
            "sample": sample,
            "slots": {f"dim{d}_{'walk' if ph == 0 else 'adjoint'}": {
                "block_threads": b[0], "blocks_per_sm": b[1], "chunk": b[2],
                "ms": {f"{c[0]}x{c[1]}x{c[2]}": round(v, 3) for c, v in slot_ms[(d, ph)].items()}}
                for (d, ph), b in slot_best.items()},
            "note": "candidates: threads per block x blocks per SM (0 = occupancy limit) x walks per queue grab; "
                    "each slot's launches timed alone"},
        "breakdown": breakdown,
        "plain_forward_points_per_s": plain,
        "plain_forward_by_dim": plain_by_dim,
        "speedup_vs_plain_forward": {k: value / v for k, v in plain.items()},
        "accuracy": {"rmse_vs_exact": (err2 / npts) ** 0.5, "rms_standard_error": (se2 / npts) ** 0.5},
        "device_status": wos.device_status(),
    }
    if compact:
        del line["breakdown"]
    if clk is not None:
        line["clocks"] = clk
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = batched_cpu_baseline(scenes, items, exact)
    plan.close()
    return line


def batched_cpu_baseline(scenes, items, exact, every=8, m=4):
    """The oracle on the host cores (all threads, LBVH) for the batched step:
    forward + adjoint of mean((u - exact)^2) on `m` points of every `every`-th
    scene, each scene with its own walk count; the per-point time of each
    sampled scene, weighted by that scene's point count, gives the workload's
    query points/s."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    adj = O.make_adj(1e-3, 0.1, True, False, 1e-3, True, True, False)
    pts, secs, walks = 0.0, 0.0, 0
    for i in range(0, len(scenes), every):
        sc, it = scenes[i], items[i]
        S = O.OracleScene(sc["V"], sc["F"], sc["g"])
        P = it.points[:m].cpu().numpy()
        n = int(it.points.shape[0])
        prm = O.make_params(nwalks=sc["nwalks"], nsteps=64, epsilon=1e-3, use_bvh=True, seed=sc["seed"])
        t0 = time.perf_counter()
        vals, _, _ = S.walk_values(P, prm, nthreads=threads)
        mean, _ = O.reduce(vals)
        S.adjoint(P, prm, adj, (2.0 * (mean - exact[i][:m]) / n).astype(np.float32), nthreads=threads)
        t = time.perf_counter() - t0
        pts += n
        secs += n * t / len(P)
        walks += len(P) * sc["nwalks"]
    return {"value": pts / secs, "unit": "points/s", "cores": threads, "kind": "port",
            "sample": f"{m} points of every {every}th scene ({walks} walks, forward + adjoint), times weighted "
                      f"by each scene's point count, {threads} threads, {cpu_info()}"}


# ---------------------------------------------------------------- 3D workload
def c3_cpu_baseline(V, F, P, npts, nw, target_s=3.0):
    """The oracle on the host cores (all threads) on bounded samples of the
    same 3D step: forward + adjoint with its binary LBVH (walks/s, the GPU
    line's unit), and the forward walk with the brute-force search (the
    reference's default)."""
    from wos import shapes
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    S = O.OracleScene(V, F, shapes.harmonic_c3(V).astype(np.float32))
    threads = os.cpu_count() or 1
    adj = O.make_adj(1e-3, 0.1, True, False, 1e-3, True, True, False)
    out = {}
    for name, bvh, with_adj, m in (("cpu_baseline", True, True, 4), ("cpu_baseline_brute_forward", False, False, 1)):
        prm = O.make_params(nwalks=nw, nsteps=64, epsilon=1e-3, use_bvh=bvh, seed=0)
        while True:
            sub = P[:m]
            t0 = time.perf_counter()
            vals, _, _ = S.walk_values(sub, prm, nthreads=threads)
            if with_adj:
                mean, _ = O.reduce(vals)
                S.adjoint(sub, prm, adj, (2.0 * mean / npts).astype(np.float32), nthreads=threads)
            tc = time.perf_counter() - t0
            if tc > target_s / 4 or m >= 4096:
                break
            m *= 4
        what = "forward + adjoint" if with_adj else "forward only, brute-force search"
        out[name] = {"value": m * nw / tc, "unit": "walks/s", "cores": threads, "kind": "port",
                     "sample": f"{m} of {npts} points x {nw} walks ({what}), {threads} threads, {cpu_info()}"}
    return out


def c3_main(args):
    print(json.dumps(c3_line(args)), flush=True)
    return 0


def c3_line(args, compact=False):
    """The 3D forward + adjoint solve: icosphere subdivided to 81,920
    triangles, radially displaced by 0.15 x seeded 3-octave value noise,
    g = x^2 - y^2 + z, seeded uniform interior points (1,000,000 by default),
    128 walks per point, nsteps 64, epsilon 1e-3; a step is the fused forward
    solve plus the adjoint of mean(u^2) with respect to vertex positions and
    per-vertex g (epsilon2 1e-3, clamping 0.1).  `compact` (the entry in the
    default bench line): the warm-up steps run on 200,000 of the points with
    16 walks each (the same scene and kernels, a quarter second per step
    instead of ten), and the untimed work-counting pass is left out."""
    import torch
    import wos
    from wos import shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F = shapes.displaced_icosphere(6, 0.15, seed=0)
    scene = NativeScene(V, F, shapes.harmonic_c3(V).astype(np.float32))
    npts, nw = args.points, args.walks if args.walks is not None else 128
    cand = shapes.sample_interior_3d(int(npts * 1.1) + 1024, shapes.displaced_radius_fn(0.15, 0), seed=1,
                                     margin=0.005)
    ins = scene.closest(cand, True, want=("inside",))["inside"].cpu().numpy().astype(bool)
    P = torch.tensor(cand[ins][:npts], device=dev)
    npts = int(P.shape[0])
    adj = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=False)

    def ws(seed):
        return WalkSettings(nwalks=nw, nsteps=64, epsilon=1e-3, seed=seed)

    warm_P, warm_nw = (P[:200_000].contiguous(), min(nw, 16)) if compact else (P, nw)
    for w in range(args.warmup):
        scene.solve_adjoint(warm_P, WalkSettings(nwalks=warm_nw, nsteps=64, epsilon=1e-3, seed=100 + w), adj,
                            loss_kind=1)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(None)
    clocks.start()
    t = 0.0
    for k in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        scene.solve_adjoint(P, ws(k), adj, loss_kind=1)
        b.record()
        torch.cuda.synchronize()
        t += a.elapsed_time(b) * 1e-3
    clk = clocks.stop()
    # forward alone, the plain kernel, accuracy and truncation on the same points
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    mean, var = scene.solve(P, ws(0), want_var=True)
    b.record()
    torch.cuda.synchronize()
    t_fwd = a.elapsed_time(b) * 1e-3
    err = mean.cpu().numpy() - shapes.harmonic_c3(P.cpu().numpy())
    se = np.sqrt(var.cpu().numpy() / nw)
    m = min(npts, max(1, (1 << 18) // nw))
    _, steps = scene.values(P[:m], ws(0), want_steps=True)
    scene.values(P[:m], ws(1), plain=True)  # untimed: the kernel's first launch loads it
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    scene.values(P[:m], ws(0), plain=True)
    b.record()
    torch.cuda.synchronize()
    t_plain = a.elapsed_time(b) * 1e-3
    # tree work of one forward solve and one fused step (device counters, untimed)
    fwd_work = fused_work = None
    if not compact:
        wos.set_work_counting(True)
        wos.work_counters(reset=True)
        scene.solve(P, ws(1))
        torch.cuda.synchronize()
        fwd_work = wos.work_counters(reset=True)
        scene.solve_adjoint(P, ws(1), adj, loss_kind=1)
        torch.cuda.synchronize()
        fused_work = wos.work_counters(reset=True)
        wos.set_work_counting(False)
    walks = npts * nw
    line = {
        "metric": "wos_walks_per_s", "value": walks * args.steps / t, "unit": "walks/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"3d_forward_adjoint_icosphere81920_pts{npts}_walks{nw}", "points": npts,
                   "walks_per_point": nw, "nsteps": 64, "epsilon": 1e-3, "epsilon2": 1e-3,
                   "loss": "mean(u^2); adjoint wrt vertex xyz and g", "nearest": "LBVH",
                   "l2": "256 MiB buffer written between timed steps (L2 flush)"},
        "adjoint_pts_per_s": npts * args.steps / t,
        "forward_walks_per_s": walks / t_fwd,
        "plain_forward_walks_per_s": m * nw / t_plain,
        "tree_work": {"forward": fwd_work, "forward_and_adjoint": fused_work,
                      "note": "queries, node expansions, leaf steps (one warp step each)"},
        "accuracy": {"rmse_vs_exact": float(np.sqrt((err ** 2).mean())), "rms_standard_error":
                     float(np.sqrt((se ** 2).mean())),
                     "truncated_fraction": float((steps.cpu().numpy() >= 64).mean())},
        "walk_steps": walk_steps(steps, 64),
        "device_status": wos.device_status(),
    }
    if compact:
        del line["tree_work"]
        line["warmup_workload"] = f"{int(warm_P.shape[0])} of the points x {warm_nw} walks"
    if clk is not None:
        line["clocks"] = clk
    if not args.no_cpu_baseline:
        line.update(c3_cpu_baseline(V, F, P.cpu().numpy(), npts, nw))
    return line


# ---------------------------------------------------------------- inverse workload
def inverse_run(scene, P, target, iters, nwalks, lr, dev, g0=None):
    """Recover per-vertex Dirichlet values from interior observations: Adam
    on g, each iteration one fused forward + adjoint of mean((u - target)^2)
    with seed = iteration (diff-wos inv_solve loop).  Returns (g, losses)."""
    import torch
    from wos.native import AdjointSettings, WalkSettings
    g = torch.zeros(scene.nV, dtype=torch.float32, device=dev) if g0 is None else g0.clone()
    g.requires_grad_(True)
    opt = torch.optim.Adam([g], lr=lr)
    adj = AdjointSettings(epsilon2=1e-3, clamping=0.1, want_dV=False, want_dg=True, want_dsrc=False)
    losses = []
    for it in range(iters):
        s = WalkSettings(nwalks=nwalks, nsteps=64, epsilon=1e-3, seed=it)
        out = scene.solve_adjoint(P, s, adj, loss_kind=2, target=target)
        losses.append(out["loss"])
        opt.zero_grad(set_to_none=False)
        g.grad = out["dg"]
        opt.step()
        with torch.no_grad():
            scene.update_values(g.detach())
    return g.detach(), torch.cat(losses)


def c1_main(args):
    """The plain 2D primal solve: unit circle as a CCW polyline of 1024 equal
    segments, g = x^3 - 3 x y^2 (harmonic, so u = g inside), no source; the
    128^2 grid on [-0.9, 0.9]^2 masked to the interior (14,592 points), 64
    walks per point, epsilon 1e-3, seed 0, nsteps 32 (and 256, reported
    beside).  A step is the solve (walks + per-point FP64 mean / variance).
    Beside it: RMSE against the closed form, the reference-shaped plain kernel
    with LBVH and brute-force search, and the oracle on the host cores in both
    search modes on a bounded sample."""
    import torch
    import wos
    from wos import shapes
    from wos.native import NativeScene, WalkSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F = shapes.circle(1024, 1.0)
    g = shapes.harmonic_c1(V).astype(np.float32)
    P = shapes.grid(128, -0.9, 0.9)
    P = np.ascontiguousarray(P[(P.astype(np.float64) ** 2).sum(1) < 1.0]).astype(np.float32)
    scene = NativeScene(V, F, g)
    Pd = torch.as_tensor(P, device=dev)
    n, nw = len(P), args.walks if args.walks is not None else 64
    exact = shapes.harmonic_c1(P)

    def ws(nsteps, seed, bvh=True):
        return WalkSettings(nwalks=nw, nsteps=nsteps, epsilon=1e-3, seed=seed, use_bvh=bvh)

    def timed(fn, reps):
        for w in range(max(3, args.warmup)):
            fn(w)
        torch.cuda.synchronize()
        t = 0.0
        for k in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn(1000 + k)
            b.record()
            torch.cuda.synchronize()
            t += a.elapsed_time(b) * 1e-3
        return t

    clocks = ClockSampler(None)
    clocks.start()
    t32 = timed(lambda k: scene.solve(Pd, ws(32, k)), args.steps)
    clk = clocks.stop()
    t256 = timed(lambda k: scene.solve(Pd, ws(256, k)), args.steps)
    accuracy = {}
    for ns in (32, 256):
        mean, var = scene.solve(Pd, ws(ns, 0), want_var=True)
        err = mean.cpu().numpy() - exact
        accuracy[f"nsteps{ns}"] = {"rmse_vs_exact": float(np.sqrt((err ** 2).mean())),
                                   "rms_standard_error": float(np.sqrt((var.cpu().numpy() / nw).mean()))}
    _, st = scene.values(Pd, ws(32, 0), want_steps=True)
    plain = {}
    for name, bvh in (("lbvh", True), ("brute", False)):
        tp = timed(lambda k: scene.values(Pd, ws(32, k, bvh), plain=True), 1)
        plain[name + "_walks_per_s"] = n * nw / tp
    # the oracle on the host cores, both search modes, bounded samples
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    S = O.OracleScene(V, F, g)
    threads = os.cpu_count() or 1
    cpu = {}
    for name, bvh in (("bvh", True), ("brute", False)):
        prm = O.make_params(nwalks=nw, nsteps=32, epsilon=1e-3, use_bvh=bvh, seed=0)
        m = 64
        while True:
            sub = P[np.linspace(0, n - 1, m).astype(np.int64)]
            t0 = time.perf_counter()
            S.walk_values(sub, prm, nthreads=threads)
            tc = time.perf_counter() - t0
            if tc > 2.0 or m >= n:
                break
            m = min(n, m * 4)
        cpu[name] = {"value": m * nw / tc, "unit": "walks/s", "cores": threads, "kind": "port",
                     "sample": f"{m} of {n} points x {nw} walks, nsteps 32, {threads} threads, {cpu_info()}"}
    walks = n * nw
    line = {
        "metric": "wos_walks_per_s", "value": walks * args.steps / t32, "unit": "walks/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t32 / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"2d_primal_circle1024_grid128_walks{nw}", "points": n, "walks_per_point": nw,
                   "nsteps": 32, "epsilon": 1e-3, "nearest": "LBVH",
                   "l2": "inputs and scene (< 1 MB) stay in L2; every step reruns the same solve"},
        "nsteps256_walks_per_s": walks * args.steps / t256,
        "plain_kernel": plain,
        "accuracy": accuracy,
        "walk_steps": walk_steps(st, 32),
        "cpu_baseline": cpu["bvh"],
        "cpu_baseline_brute": cpu["brute"],
        "device_status": wos.device_status(),
    }
    if clk is not None:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    return 0


def fd_check(make_scene, V, P_d, settings, adjoint, seeds, nvert=32, hs=(1e-3, 5e-4)):
    """Vertex gradient of loss = mean(u^2) from the fused forward + adjoint
    step against central finite differences with common random numbers (the
    same seed on both sides), along seeded random directions at `nvert`
    seeded random vertices, over `seeds` seeds; per vertex and step h the
    z-score of (adjoint - FD) against the seed-to-seed standard errors of
    both."""
    import torch
    dim = V.shape[1]
    rng = np.random.default_rng(1)
    ks = rng.choice(len(V), nvert, replace=False)
    dirs = rng.normal(size=(nvert, dim))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    base, moved = make_scene(), make_scene()
    adj = np.zeros((seeds, nvert))
    fd = np.zeros((len(hs), seeds, nvert))
    t0 = time.perf_counter()
    for si in range(seeds):
        s = settings(500 + si)
        adj[si] = (base.solve_adjoint(P_d, s, adjoint, loss_kind=1)["dV"].cpu().numpy()[ks] * dirs).sum(1)
        for j, (k, d) in enumerate(zip(ks, dirs)):
            for hi, h in enumerate(hs):
                loss = []
                for sign in (1.0, -1.0):
                    Vm = V.copy()
                    Vm[k] += sign * h * d
                    moved.update_vertices(torch.as_tensor(Vm, device=P_d.device))
                    loss.append(float((moved.solve(P_d, s) ** 2).mean()))
                fd[hi, si, j] = (loss[0] - loss[1]) / (2 * h)
    t = time.perf_counter() - t0
    checks = {}
    for hi, h in enumerate(hs):
        se = np.sqrt(adj.var(0, ddof=1) / seeds + fd[hi].var(0, ddof=1) / seeds)
        z = (adj.mean(0) - fd[hi].mean(0)) / np.maximum(se, 1e-30)
        checks[f"h{h:g}"] = {"within_2se": float(np.mean(np.abs(z) < 2.0)), "max_abs_z": float(np.abs(z).max()),
                             "z": [float(x) for x in z], "fd_mean": [float(x) for x in fd[hi].mean(0)],
                             "se": [float(x) for x in se]}
    return t, {"vertices": [int(k) for k in ks], "adjoint_mean": [float(x) for x in adj.mean(0)],
               "checks": checks}


def fd_line(workload, npts, seeds, t, res, note, hs, eps):
    h0 = f"h{hs[0]:g}"
    return {
        "metric": "vertex_gradient_fd_check", "value": res["checks"][h0]["within_2se"],
        "unit": f"fraction of vertices within 2 SE (h = {hs[0]:g})", "n_gpus": 1, "steps": seeds, "warmup": 0,
        "ms_per_step": t / seeds * 1e3, "higher_is_better": True, "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload, "points": npts, "points_note": note, "h": list(hs), "epsilon": eps,
                   "seeds": seeds, "fd": "central, common random numbers"},
        **res,
    }


def fd_main(args):
    """The 2D differentiable solve's gradient check (fd_check) at 32 vertices,
    h = 1e-3 as specified and h = 5e-4.  With h equal to the termination
    shell epsilon (1e-3), a move changes which walks end in the shell, so
    where the normal derivative is large the loss is visibly nonlinear at
    that scale and the h = 1e-3 difference is biased; h = 5e-4 shows the
    estimate converging to the adjoint.  Query points within 0.01 of the
    boundary are left out: a vertex moved by h can carry such a point outside
    the domain, which ends its walks (value 0) -- a jump of the loss that the
    finite difference sees and the shape derivative of the fixed point set
    does not."""
    import torch
    from wos import shapes
    from wos.native import NativeScene
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F, g, P = make_workload()
    P = np.ascontiguousarray(P[shapes.inside_star(P, STAR["r0"], STAR["amp"], STAR["lobes"], margin=0.01)])
    t, res = fd_check(lambda: NativeScene(V, F, g, 2, SOURCE), V, torch.as_tensor(P, device=dev), walk_settings,
                      adjoint_settings(), args.seeds, hs=args.fd_h)
    print(json.dumps(fd_line(workload_config(len(P))["workload"], len(P), args.seeds, t, res,
                             "grid points at least 0.01 inside the boundary", args.fd_h, EPS)), flush=True)
    return 0


def c3fd_main(args):
    """The 3D solve's gradient check (fd_check) on the displaced icosphere
    (81,920 triangles, g = x^2 - y^2 + z) at 32 vertices, 20,000 seeded
    interior points at least 0.01 inside (radially), 128 walks, epsilon 1e-3."""
    import torch
    from wos import shapes
    from wos.native import AdjointSettings, NativeScene, WalkSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F = shapes.displaced_icosphere(6, 0.15, seed=0)
    g = shapes.harmonic_c3(V).astype(np.float32)
    P = shapes.sample_interior_3d(20000, shapes.displaced_radius_fn(0.15, 0), seed=2, margin=0.01)
    P = np.ascontiguousarray(P[:20000]).astype(np.float32)
    adj = AdjointSettings(epsilon2=EPS2, clamping=0.1, want_dV=True, want_dg=True, want_dsrc=False)

    def ws(seed):
        return WalkSettings(nwalks=128, nsteps=64, epsilon=EPS, seed=seed)

    t, res = fd_check(lambda: NativeScene(V, F, g), V, torch.as_tensor(P, device=dev), ws, adj, args.seeds,
                      hs=args.fd_h)
    print(json.dumps(fd_line("3d_forward_adjoint_icosphere81920_pts20000_walks128", len(P), args.seeds, t, res,
                             "seeded interior points at least 0.01 inside (radially)", args.fd_h, EPS)), flush=True)
    return 0


def c4_main(args):
    """The 2D inverse problem: star r = 0.6 + 0.25 cos 5 theta with 8192
    segments, unknown per-vertex g (initialised to 0), target = the solve with
    g* = cos 4 theta + 0.5 sin 7 theta on the 256^2 grid masked to the
    interior (19,988 points; 1024 walks, untimed); `--iters` Adam iterations
    (lr 1e-2) of 32 walks per point, each a fused forward + adjoint step."""
    import torch
    import wos
    from wos import shapes
    from wos.native import NativeScene, WalkSettings
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F = shapes.star(8192, 0.6, 0.25, 5)
    th = np.arctan2(V[:, 1], V[:, 0]).astype(np.float64)
    g_true = (np.cos(4 * th) + 0.5 * np.sin(7 * th)).astype(np.float32)
    P = shapes.grid(256, -1.0, 1.0)
    P = P[shapes.inside_star(P, 0.6, 0.25, 5)]
    Pd = torch.as_tensor(np.ascontiguousarray(P), device=dev)
    truth = NativeScene(V, F, g_true)
    target = truth.solve(Pd, WalkSettings(nwalks=1024, nsteps=64, epsilon=1e-3, seed=12345)).to(torch.float32)
    scene = NativeScene(V, F, np.zeros_like(g_true))
    # warm-up iterations, then the unknowns start again from zero
    inverse_run(scene, Pd, target, args.warmup, 32, 1e-2, dev)
    scene.update_values(torch.zeros(len(g_true), device=dev))
    torch.cuda.synchronize()
    clocks = ClockSampler(None)
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    g, losses = inverse_run(scene, Pd, target, args.iters, 32, 1e-2, dev)
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = a.elapsed_time(b) * 1e-3
    losses = losses.cpu().numpy()
    gt = torch.as_tensor(g_true, device=dev)
    walks = len(P) * 32
    line = {
        "metric": "wos_walks_per_s", "value": walks * args.iters / t, "unit": "walks/s", "n_gpus": 1,
        "steps": args.iters, "warmup": args.warmup, "ms_per_step": t / args.iters * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "2d_inverse_values_star8192_grid256_walks32", "points": len(P), "walks_per_point": 32,
                   "iterations": args.iters, "optimizer": "Adam lr 1e-2", "loss": "mean((u - target)^2)",
                   "nsteps": 64, "epsilon": 1e-3,
                   "timed": "the whole optimisation loop: fused step, Adam update, scene value update"},
        "iterations_per_s": args.iters / t,
        "loss_first": float(losses[0]), "loss_last10_mean": float(losses[-10:].mean()),
        "g_rel_error": float(torch.linalg.norm(g - gt) / torch.linalg.norm(gt)),
        "device_status": wos.device_status(),
    }
    if clk is not None:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="leave the 3D and batched entries out of the default 2D line")
    ap.add_argument("--ref-step-s", type=float, default=6.0)
    ap.add_argument("--grid", type=int, default=GRID, help="query grid (smaller only for profiling captures)")
    ap.add_argument("--walks", type=int, default=None,
                    help="walks per point (c2: 256, c3: 128; smaller only for profiling)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c2fd", "c3", "c3fd", "c4", "batched"],
                    help="c2: the 2D differentiable solve (default); c1: the plain 2D primal solve; "
                         "c2fd / c3fd: vertex gradients against finite differences; "
                         "c3: the 3D forward + adjoint solve; c4: the 2D inverse problem; "
                         "batched: many scenes in one launch")
    ap.add_argument("--seeds", type=int, default=16, help="seeds of the c2fd gradient check")
    ap.add_argument("--fd-h", default="1e-3,5e-4", help="c2fd / c3fd: comma-separated finite-difference steps")
    ap.add_argument("--fd-eps", type=float, default=None,
                    help="c2fd / c3fd: termination shell epsilon of the walks and the ball walks (default 1e-3)")
    ap.add_argument("--iters", type=int, default=500, help="Adam iterations of the c4 workload")
    ap.add_argument("--points", type=int, default=1_000_000, help="query points of the c3 workload")
    ap.add_argument("--scale", type=float, default=0.1, help="query-count scale of the batched workload")
    args = ap.parse_args()
    set_size(args.grid, args.walks if args.walks is not None else NWALKS)
    args.fd_h = tuple(float(x) for x in args.fd_h.split(","))
    if args.fd_eps is not None:
        global EPS, EPS2
        EPS = EPS2 = float(args.fd_eps)
    if args.workload == "batched" and args.impl == "ours":
        return batched_main(args)
    if args.workload == "c1" and args.impl == "ours":
        return c1_main(args)
    if args.workload == "c2fd" and args.impl == "ours":
        return fd_main(args)
    if args.workload == "c3fd" and args.impl == "ours":
        return c3fd_main(args)
    if args.workload == "c3" and args.impl == "ours":
        return c3_main(args)
    if args.workload == "c4" and args.impl == "ours":
        return c4_main(args)
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, world, rank)

    import torch
    import torch.distributed as dist
    import wos
    from wos.native import NativeScene

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    V, F, g, P = make_workload()
    n = len(P)
    dev = torch.device("cuda", local)
    scene = NativeScene(V, F, g, 2, SOURCE)
    P_d = torch.as_tensor(P, device=dev)
    ws = walk_settings(seed=1000 * rank)
    adj = adjoint_settings()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    import ctypes
    from wos import _lib
    c = ws.c()
    ca = adj.c()
    fused_ws = torch.empty(_lib.lib().wos_solve_adjoint_workspace_size(scene.h, n, ctypes.byref(c), ctypes.byref(ca)),
                           dtype=torch.uint8, device=dev)
    solve_ws = torch.empty(_lib.lib().wos_solve_workspace_size(n, ctypes.byref(c)), dtype=torch.uint8, device=dev)
    adj_ws = torch.empty(_lib.lib().wos_adjoint_records_workspace_size(scene.h, n, ctypes.byref(c)),
                         dtype=torch.uint8, device=dev)

    def step(seed):
        """One fused forward + adjoint step (wos_solve_adjoint, loss = mean(u^2))."""
        return scene.solve_adjoint(P_d, walk_settings(seed), adj, loss_kind=1, workspace=fused_ws)

    def split_step(seed, times):
        """The same kernels as separate calls, for the per-kernel breakdown."""
        s = walk_settings(seed)
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(stream)
        mean, _, rec, dc = scene.solve_records(P_d, s, want_dcontrib=True, workspace=solve_ws)
        e1.record(stream)
        dLdu = (2.0 / n) * mean.to(torch.float32)
        scene.adjoint_records(P_d, s, adj, dLdu, rec, dc, workspace=adj_ws)
        e2.record(stream)
        times.append((e0, e1, e2))

    # -- work counting pass (untimed): exact tree work of one step's launches
    wos.set_work_counting(True)
    _lib.work_counters(reset=True)
    s0 = walk_settings(7)
    mean0, _, rec0, dc0 = scene.solve_records(P_d, s0, want_dcontrib=True, workspace=solve_ws)
    torch.cuda.synchronize()
    fwd_work = _lib.work_counters(reset=True)
    scene.adjoint_records(P_d, s0, adj, (2.0 / n) * mean0.to(torch.float32), rec0, dc0, workspace=adj_ws)
    torch.cuda.synchronize()
    adj_work = _lib.work_counters(reset=True)
    wos.set_work_counting(False)
    del rec0, dc0

    # -- warm-up
    for w in range(args.warmup):
        step(10_000 + w)
    torch.cuda.synchronize()
    wos.device_status(reset=True)

    # -- timed steps (device), L2 flushed between steps
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_times = []
    for k in range(args.steps):
        flush.zero_()
        e0, e1 = ev(), ev()
        e0.record(stream)
        step(1000 * rank + k)
        e1.record(stream)
        step_times.append((e0, e1))
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    t_step = float(sum(a.elapsed_time(b) for a, b in step_times)) * 1e-3
    t_max = max_over_ranks(t_step)
    status = wos.device_status(reset=False)

    # -- per-kernel breakdown (separate, untimed for `value`)
    times = []
    for k in range(max(2, min(args.steps, 3))):
        flush.zero_()
        split_step(2000 + k, times)
    torch.cuda.synchronize()
    t_solve = [a.elapsed_time(b) * 1e-3 for a, b, _ in times]
    t_adj = [b.elapsed_time(c) * 1e-3 for _, b, c in times]

    total_walks = world * n * NWALKS * args.steps
    value = total_walks / t_max
    ms_per_step = t_max / args.steps * 1e3

    # -- e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = e2e_bench(args, V, F, g, P, rank, world, dev, max_over_ranks, barrier)

    # -- plain (reference-shaped) forward kernel vs the persistent one, same walks
    plain = plain_vs_persistent(scene, P_d, n)
    # -- steps per walk on a sample of points spread over the grid (untimed)
    stride = max(1, n // max(1, (1 << 18) // NWALKS))
    _, st = scene.values(P_d[::stride].contiguous(), walk_settings(3), want_steps=True)
    steps_stats = walk_steps(st, NSTEPS)

    hbm, peak_kind = peaks()
    adj_avg = float(np.mean(t_adj))
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6
    traffic = None
    ipq = None
    tj = {}
    tp = ROOT / "profiles" / "roofline_traffic.json"
    if tp.exists():
        tj = json.load(open(tp))
        if tj.get("kernel") == "k_adjoint" and tj.get("workload") == workload_config(n)["workload"]:
            traffic = tj.get("traffic_bytes_per_launch")
            ipq = tj.get("warp_instructions_per_query")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(n),
        "adjoint_pts_per_s": world * n * args.steps / t_max,
        "breakdown_ms": {"forward_kernel_and_reduce": float(np.mean(t_solve)) * 1e3, "adjoint": adj_avg * 1e3,
                         "note": "separate calls of the fused step's kernels"},
        "gpu_launches": args.steps * fused_step_launches(len(F)),
        "device_status": status,
        "plain_vs_persistent": plain,
        "walk_steps": steps_stats,
        "tree_work_per_launch": {"adjoint": adj_work, "forward": fwd_work,
                                 "note": "this build's wide-tree counters: queries, node expansions and leaf "
                                         "steps (one warp step each)"},
    }
    if clk is not None:
        line["clocks"] = clk
    if e2e is not None:
        line["e2e"] = e2e
    # issue roofline of the adjoint kernel: warp instructions per nearest
    # query (ncu capture of the same kernel) x this launch's queries (device
    # counters) / its CUDA-event time, against one warp instruction per cycle
    # on each of the 4 schedulers of 148 SMs at the median SM clock
    issue_peak = 148 * 4 * sm_mhz * 1e6
    if ipq is not None:
        inst = float(ipq) * adj_work["queries"]
        line["roofline"] = {
            "bound": "issue", "achieved": inst / adj_avg / 1e9, "peak": issue_peak / 1e9, "unit": "Ginst/s",
            "frac": inst / adj_avg / issue_peak, "traffic": traffic, "kernel": "k_adjoint",
            "peak_kind": f"148 SMs x 4 warp schedulers x {sm_mhz:.0f} MHz (median SM clock of the timed region)",
            "per_unit": {"unit": "nearest query (one warp-cooperative wide-tree search)",
                         "warp_instructions_per_query": ipq, "queries_per_launch": adj_work["queries"],
                         "source": tj.get("instructions_measured_on")},
            "note": "the scene and trees (~0.2 MB) stay in L1/L2 and DRAM traffic is the per-walk records "
                    "(`traffic`, bytes per launch); the kernel is bound by instruction issue",
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        S, prm, adjp, run, m, threads = cpu_baseline(V, F, g, P)
        ts = [run(m) for _ in range(2)]
        tcpu = float(np.mean(ts))
        line["cpu_baseline"] = {"value": m * NWALKS / tcpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{m} of {n} points x {NWALKS} walks (forward + adjoint), "
                                          f"{threads} threads, {cpu_info()}"}
        line["accuracy"] = fp64_accuracy(scene, V, F, g, P, P_d, threads)
        # roofline of the adjoint kernel on the reference algorithm's work
        ref = reference_work(S, prm, adjp, P)
        samples = n * NWALKS
        adj_bytes, adj_ops = algorithmic({k: v * samples for k, v in ref["adjoint"].items()})
        achieved = adj_bytes / adj_avg / 1e9
        line.setdefault("roofline", {"bound": "issue", "achieved": None, "peak": issue_peak / 1e9,
                                     "unit": "Ginst/s", "frac": None, "traffic": traffic, "kernel": "k_adjoint"})
        line["roofline"]["ref_lbvh_bytes"] = {
            "achieved_gbs": achieved, "peak_gbs": hbm, "peak_kind": peak_kind, "frac": achieved / hbm,
            "algorithmic_bytes_per_launch": adj_bytes,
            "per_unit": {"unit": "adjoint sample (one walk's boundary-shape + normal-derivative estimate)",
                         "reference_lbvh_work": ref["adjoint"], "forward_walk_work": ref["forward"],
                         "sample": ref["sample"]},
            "note": "the reference binary LBVH traversal's box and primitive reads for the same samples, over "
                    "the HBM copy peak; they are served from L1/L2, not HBM",
        }
        line["roofline"]["fp32_algorithmic"] = {"achieved_tflops": adj_ops / adj_avg / 1e12,
                                                "peak_tflops": fp32_peak / 1e12, "frac": adj_ops / adj_avg / fp32_peak}
    if rank == 0 and world == 1 and not args.no_other_workloads:
        line["other_workloads"] = other_workloads(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def other_workloads(args):
    """The configured 3D and batched workloads, run after the 2D step's line
    is complete and reported beside it (one GPU): the displaced icosphere at
    1,000,000 points x 128 walks, and the 256-scene batch at full scale, each
    with its own warm-up, CUDA-event timing, clocks, accuracy against the exact
    solutions and CPU baseline.  Neither touches the 2D line's figures."""
    import gc
    import torch
    out = {}
    jobs = (("c3_3d_forward_adjoint", c3_line, dict(points=1_000_000, walks=128, steps=2, warmup=3)),
            ("c5_batched", batched_line, dict(scale=1.0, steps=1, warmup=1)))
    for name, fn, kw in jobs:
        ns = argparse.Namespace(**{**vars(args), **kw})
        t0 = time.perf_counter()
        try:
            out[name] = fn(ns, compact=True)
        except Exception as e:  # the 2D line is printed whatever happens here
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = round(time.perf_counter() - t0, 1)
        gc.collect()
        try:
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        except Exception:
            pass
    return out


def fused_step_launches(nF: int) -> int:
    """This library's kernel launches in one fused wos_solve_adjoint step
    (dV, dg and dsrc wanted, sample order on): k_walk, k_reduce, k_loss,
    k_prim_rank, k_record_keys, the radix sort's histogram and prefix-sum
    kernels plus one onesweep pass per 8 key bits (keys up to nF), k_adjoint,
    and three k_add_f64_to_f32."""
    bits = 1
    while bits < 32 and (1 << bits) <= nF:
        bits += 1
    return 9 + 2 + (bits + 7) // 8


def fp64_accuracy(scene, V, F, g, P, P_d, threads, npts=256, ref_walks=16384):
    """Error of the solve against an FP64 solution.  The star with f = 1 has
    no closed form, so the reference is the oracle's double-precision
    walk-on-spheres (source term by its expectation R^2 / 4 per step) at
    ref_walks walks on npts points spread over the grid; the GPU solve runs at
    the bench's walk count on the same points.  RMSE ~ sqrt(SE_gpu^2 +
    SE_ref^2) when both are unbiased."""
    import torch
    from oracle import oracle as O
    idx = np.linspace(0, len(P) - 1, npts).astype(np.int64)
    S = O.OracleScene(V, F, g)
    ref_mean, ref_var, ref_trunc = S.solve_f64(P[idx], ref_walks, 1.0, eps=EPS, seed=424242, nthreads=threads)
    mean, var = scene.solve(P_d[torch.as_tensor(idx, device=P_d.device)], walk_settings(11), want_var=True)
    mean, var = mean.cpu().numpy(), var.cpu().numpy()
    se = float(np.sqrt((var / NWALKS).mean()))
    se_ref = float(np.sqrt((ref_var / ref_walks).mean()))
    return {"rmse_vs_fp64": float(np.sqrt(((mean - ref_mean) ** 2).mean())), "rms_standard_error": se,
            "expected_rmse": float(np.hypot(se, se_ref)),
            "fp64_reference": {"points": npts, "walks": ref_walks, "rms_standard_error": se_ref,
                               "truncated_walks": ref_trunc,
                               "estimator": "oracle FP64 walk-on-spheres, source term R^2/4 per step"}}


def walk_steps(steps, nsteps):
    """Steps-per-walk statistics of a sample of walks: quantiles, a histogram
    over power-of-two bins, and the fraction truncated at nsteps."""
    s = steps.reshape(-1).cpu().numpy()
    edges = [0] + [e for e in (4, 8, 16, 32) if e < nsteps - 1] + [nsteps - 1]
    hist, lo = {}, 0
    for e in edges[1:]:
        hist[f"{lo + (1 if lo else 0)}-{e}"] = float(((s > lo) & (s <= e)).mean()) if lo else float((s <= e).mean())
        lo = e
    hist[f">={nsteps}"] = float((s >= nsteps).mean())
    return {"walks": int(s.size), "mean": float(s.mean()), "p50": float(np.percentile(s, 50)),
            "p90": float(np.percentile(s, 90)), "p99": float(np.percentile(s, 99)), "histogram": hist,
            "truncated_fraction": float((s >= nsteps).mean())}


def plain_vs_persistent(scene, P_d, n):
    """Forward-only walks/s of the reference-shaped kernel (one thread per
    walk, no regeneration) and of the persistent kernel, same walks."""
    import torch
    s = walk_settings(3)
    out = {}
    for name, plain in (("plain", True), ("persistent", False)):
        scene.values(P_d, s, plain=plain)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        scene.values(P_d, s, plain=plain)
        b.record()
        torch.cuda.synchronize()
        out[name + "_fwd_walks_per_s"] = n * NWALKS / (a.elapsed_time(b) * 1e-3)
    return out


def e2e_bench(args, V, F, g, P, rank, world, dev, max_over_ranks, barrier):
    import torch
    import wos
    Vh = torch.from_numpy(V).pin_memory()
    Fh = torch.from_numpy(F).pin_memory()
    gh = torch.from_numpy(g).pin_memory()
    Ph = torch.from_numpy(P).pin_memory()
    sh = torch.tensor(SOURCE, dtype=torch.float32).pin_memory()
    n = len(P)
    fwd = wos.WoSWithSourceCUDA(nwalks=NWALKS, nsteps=NSTEPS, epsilon=EPS, use_IS_for_greens=True)
    bwd = wos.OursCUDA(nwalks=NWALKS, nsteps=NSTEPS, epsilon=EPS, epsilon2=EPS2, clamping=CLAMP, grad_values=True,
                       grad_source=True, use_IS_for_greens=True)
    solver = wos.CustomSolver(fwd_solver=fwd, bwd_solver=bwd)
    h2d = Vh.numel() * 4 + Fh.numel() * 4 + gh.numel() * 4 + Ph.numel() * 4 + sh.numel() * 4
    d2h = 4 + Vh.numel() * 4 + gh.numel() * 4 + sh.numel() * 4

    def one(seed):
        Vd = Vh.to(dev, non_blocking=True).requires_grad_(True)
        gd = gh.to(dev, non_blocking=True).requires_grad_(True)
        sd = sh.to(dev, non_blocking=True).requires_grad_(True)
        Pd = Ph.to(dev, non_blocking=True)
        scene = wos.Polyline(Vd, Fh.to(dev, non_blocking=True), gd, source_type=2, source_params=sd, use_bvh=True)
        u = solver.walk(Pd, scene, seed=seed)
        loss = (u * u).mean()
        loss.backward()
        return loss.detach().cpu(), Vd.grad.cpu(), gd.grad.cpu(), sd.grad.cpu()

    for w in range(args.warmup):
        one(20_000 + w)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        one(30_000 + 1000 * rank + k)
    e1.record()
    torch.cuda.synchronize()
    t = max_over_ranks(e0.elapsed_time(e1) * 1e-3)
    return {"value": world * n * NWALKS * args.steps / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": t / args.steps * 1e3,
            "path": "wos.CustomSolver(WoSWithSourceCUDA, OursCUDA).walk + torch autograd, pinned host buffers"}


if __name__ == "__main__":
    sys.exit(main())
