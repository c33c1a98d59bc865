"""Batched forward + adjoint over many scenes in one persistent launch per
dimension, replayed as one CUDA graph (wos_batch_* in the C ABI)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import WosAdjointParams, WosBatchItem, call
from .native import AdjointSettings, NativeScene, WalkSettings, as_cuda, stream


@dataclass
class BatchItem:
    """One scene and its query points.  loss_kind 1: mean(u^2); 2:
    mean((u - target)^2); 0: target holds dL/du."""
    scene: object  # Polyline, Scene3D or NativeScene
    points: torch.Tensor
    settings: WalkSettings
    loss_kind: int = 1
    target: torch.Tensor | None = None


def _native(scene) -> NativeScene:
    return scene if isinstance(scene, NativeScene) else scene._native


class BatchPlan:
    """A planned batch.  Items keep their points / targets alive (the plan's
    graph reads them in place); order items scene-major."""

    def __init__(self, items: list[BatchItem], adjoint: AdjointSettings | None = None):
        self.items = []
        arr = (WosBatchItem * len(items))()
        for i, it in enumerate(items):
            ns = _native(it.scene)
            P = as_cuda(it.points, torch.float32, ns.dim).reshape(-1, ns.dim)
            tg = as_cuda(it.target, torch.float32).reshape(-1) if it.target is not None else None
            self.items.append((ns, P, tg, it))
            arr[i] = WosBatchItem(ns.h.value, P.data_ptr(), int(P.shape[0]), int(it.loss_kind),
                                  tg.data_ptr() if tg is not None else None, it.settings.c())
        self._adj = (adjoint or AdjointSettings()).c()
        self.want_adjoint = adjoint is not None
        h = ctypes.c_void_p()
        call("wos_batch_create", arr, len(items), ctypes.byref(self._adj), int(self.want_adjoint), stream(),
             ctypes.byref(h))
        self.h = h

    def set_launch(self, block_threads=256, blocks_per_sm=0, chunk=64):
        call("wos_batch_set_launch", self.h, int(block_threads), int(blocks_per_sm), int(chunk))

    def autotune(self, candidates, repeats: int = 1):
        """Time whole steps for each (block_threads, chunk) candidate and keep
        the fastest (wos_batch_autotune).  Returns (best, {candidate: ms})."""
        n = len(candidates)
        bt = (ctypes.c_int32 * n)(*[int(c[0]) for c in candidates])
        ch = (ctypes.c_int32 * n)(*[int(c[1]) for c in candidates])
        ms = (ctypes.c_float * n)()
        best = ctypes.c_int32()
        call("wos_batch_autotune", self.h, bt, ch, n, int(repeats), stream(), ms, ctypes.byref(best))
        cands = [tuple(int(x) for x in c) for c in candidates]
        return cands[best.value], {c: float(ms[i]) for i, c in enumerate(cands)}

    def autotune_slots(self, candidates, repeats: int = 1, sample: float = 1.0):
        """Per (dimension, phase) slot, time that slot's launches alone on the
        first `sample` fraction of its walks for each (block_threads,
        blocks_per_sm, chunk) candidate and keep the fastest
        (wos_batch_autotune_slots).  Returns ({slot: best candidate},
        {slot: {candidate: ms}}) for the slots present, slot = (dim, phase)."""
        n = len(candidates)
        bt = (ctypes.c_int32 * n)(*[int(c[0]) for c in candidates])
        bs = (ctypes.c_int32 * n)(*[int(c[1]) for c in candidates])
        ch = (ctypes.c_int32 * n)(*[int(c[2]) for c in candidates])
        ms = (ctypes.c_float * (4 * n))()
        best = (ctypes.c_int32 * 4)()
        call("wos_batch_autotune_slots", self.h, bt, bs, ch, n, int(repeats), float(sample), stream(), ms, best)
        cands = [tuple(int(x) for x in c) for c in candidates]
        chosen, times = {}, {}
        for k in range(4):
            if best[k] < 0:
                continue
            slot = (2 + k // 2, k % 2)
            chosen[slot] = cands[best[k]]
            times[slot] = {c: float(ms[k * n + i]) for i, c in enumerate(cands)}
        return chosen, times

    def set_launch_slot(self, dim: int, phase: int, block_threads=256, blocks_per_sm=0, chunk=64):
        call("wos_batch_set_launch_slot", self.h, int(dim), int(phase), int(block_threads), int(blocks_per_sm),
             int(chunk))

    def launch(self, dim: int, phase: int):
        """(block_threads, blocks_per_sm, chunk) of slot (dim, phase)."""
        out = (ctypes.c_int32 * 3)()
        call("wos_batch_get_launch", self.h, int(dim), int(phase), out)
        return tuple(int(x) for x in out)

    def refresh(self):
        """Re-read the scenes' device views now.  run() does this by itself
        for scenes whose vertices (NativeScene.update_vertices) or source
        changed since the last step, so this is rarely needed."""
        call("wos_batch_refresh", self.h, stream())

    def run(self, use_graph=True):
        call("wos_batch_run", self.h, int(use_graph), stream())

    def info(self):
        w, p, g = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        call("wos_batch_info", self.h, ctypes.byref(w), ctypes.byref(p), ctypes.byref(g))
        return dict(walks=int(w.value), points=int(p.value), groups=int(g.value))

    def outputs(self, i):
        ns, P, _, _ = self.items[i]
        n = int(P.shape[0])
        d = P.device
        mean = torch.empty(n, dtype=torch.float64, device=d)
        var = torch.empty(n, dtype=torch.float64, device=d)
        loss = torch.empty(1, dtype=torch.float64, device=d)
        out = dict(mean=mean, var=var, loss=loss)
        grads = [None, None, None]
        if self.want_adjoint:
            grads = [torch.empty((ns.nV, ns.dim), dtype=torch.float32, device=d),
                     torch.empty(ns.nV, dtype=torch.float32, device=d),
                     torch.empty(5, dtype=torch.float32, device=d)]
        call("wos_batch_copy_outputs", self.h, i, mean.data_ptr(), var.data_ptr(), loss.data_ptr(),
             *[g.data_ptr() if g is not None else None for g in grads], stream())
        out.update(dV=grads[0], dg=grads[1], dsrc=grads[2])
        return out

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            try:
                _lib.lib().wos_batch_destroy(self.h, stream())
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.close()
