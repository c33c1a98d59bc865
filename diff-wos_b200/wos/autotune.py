"""Launch-shape autotuner for the persistent walk / adjoint kernels.

The knobs are the threads per block, the resident blocks per SM and the
number of walks a warp takes from the global queue per grab (chunk); a
batched plan keeps one shape per (dimension, phase) slot.  Results
never depend on them (walks are defined by their Philox counters), only speed
does.  The tuner times a few candidates on the caller's own workload with
CUDA events and keeps the fastest; results are cached per (GPU, dimension,
scene-size bucket, kind) in ~/.cache/wos_b200/autotune.json.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

import torch

from . import _lib

CANDIDATES = [(128, 32), (256, 32), (256, 64), (256, 128), (512, 64), (128, 16)]
# (threads per block, blocks per SM (0 = occupancy limit), walks per queue
# grab) for the slot-wise batch tuner: block size x grab size at full
# occupancy, plus fewer resident blocks (more L1 and shared memory per block)
SLOT_CANDIDATES = ([(b, 0, c) for b in (128, 256, 512) for c in (16, 32, 64, 128)]
                   + [(256, 2, 32), (256, 3, 32), (128, 4, 32), (128, 6, 32)])
CACHE = Path(os.environ.get("WOS_B200_CACHE", Path.home() / ".cache" / "wos_b200")) / "autotune.json"


def _key(dim: int, nF: int, kind: str) -> str:
    return f"{torch.cuda.get_device_name()}|{dim}|{int(math.log2(max(nF, 1)))}|{kind}"


def _load() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def _save(d: dict) -> None:
    try:
        CACHE.parent.mkdir(parents=True, exist_ok=True)
        CACHE.write_text(json.dumps(d, indent=1))
    except OSError:
        pass


def _time(fn, repeats: int) -> float:
    fn()  # first call compiles nothing but touches caches / allocator
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune_scene(native, P, settings, adjoint=None, candidates=None, repeats: int = 2, use_cache: bool = True):
    """Pick the launch shape for `native`'s dimension on this workload (the
    fused forward + adjoint step if `adjoint` is given, else the solve) and
    set it with wos_set_launch_config.  Returns (config, {config: ms})."""
    kind = "fused" if adjoint is not None else "solve"
    key = _key(native.dim, native.nF, kind)
    cache = _load() if use_cache else {}
    if key in cache:
        bt, chunk = cache[key]
        _lib.set_launch_config(native.dim, block_threads=bt, chunk=chunk)
        return (bt, chunk), {}
    old = _lib.get_launch_config(native.dim)
    times = {}
    for bt, chunk in candidates or CANDIDATES:
        _lib.set_launch_config(native.dim, block_threads=bt, chunk=chunk)
        if adjoint is not None:
            fn = lambda: native.solve_adjoint(P, settings, adjoint, loss_kind=1)  # noqa: E731
        else:
            fn = lambda: native.solve(P, settings)  # noqa: E731
        times[(bt, chunk)] = _time(fn, repeats)
    best = min(times, key=times.get)
    _lib.set_launch_config(native.dim, block_threads=best[0], blocks_per_sm=old.blocks_per_sm, chunk=best[1])
    if use_cache:
        cache[key] = list(best)
        _save(cache)
    return best, times


def tune_batch(plan, candidates=None, repeats: int = 1):
    """Pick the launch shape of a BatchPlan by timing whole steps (the
    library's wos_batch_autotune, on the current stream)."""
    return plan.autotune(candidates or CANDIDATES, repeats)


def tune_batch_slots(plan, candidates=None, repeats: int = 1, sample: float = 1.0):
    """Pick a launch shape per (dimension, phase) slot of a BatchPlan by
    timing each slot's launches alone (wos_batch_autotune_slots): block size,
    resident blocks per SM and walks per queue grab.  `sample` < 1 times a
    prefix of each run's walks, for large plans."""
    return plan.autotune_slots(candidates or SLOT_CANDIDATES, repeats, sample)
