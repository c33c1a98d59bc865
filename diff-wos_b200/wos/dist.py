"""Multi-GPU helpers: one process per GPU, torch.distributed for plumbing.

A solve shards by walks: every rank runs walks [offset, offset + count) of
every query point (Philox walk indices stay global, so the union over ranks
is exactly the single-GPU set of walks) with the scene and its trees
replicated.  The forward needs one weighted sum of per-point means, the
adjoint one sum-all-reduce of the gradient buffers (dV, dg and the 5 source
coefficients).  No kernel waits on another rank.
"""
from __future__ import annotations

import dataclasses

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(n: int, rank: int, size: int) -> tuple[int, int]:
    """Contiguous [start, end) of n items for rank out of size; sizes differ by at most one."""
    base, extra = divmod(n, size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def allreduce_sum_(tensors) -> None:
    """In-place sum over ranks of every non-None tensor (one flat float64 buffer)."""
    ts = [t for t in tensors if t is not None]
    rank, size = world()
    if size == 1 or not ts:
        return
    flat = torch.cat([t.reshape(-1).to(torch.float64) for t in ts])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    o = 0
    for t in ts:
        k = t.numel()
        t.copy_(flat[o:o + k].view_as(t).to(t.dtype))
        o += k


def max_over_ranks(x: float, device=None) -> float:
    rank, size = world()
    if size == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _local(settings, rank, size):
    a, b = shard(int(settings.nwalks), rank, size)
    return dataclasses.replace(settings, walk_offset=int(settings.walk_offset) + a, nwalks=b - a), b - a


def sharded_solve(native_scene, P, settings):
    """Per-point means over all nwalks walks, this rank running its share."""
    rank, size = world()
    local, count = _local(settings, rank, size)
    if count > 0:
        mean = native_scene.solve(P, local) * (count / settings.nwalks)
    else:
        mean = torch.zeros(P.shape[0], dtype=torch.float64, device=P.device)
    allreduce_sum_([mean])
    return mean


def sharded_adjoint(native_scene, P, settings, adjoint, dLdu):
    """Gradients of sum_i dLdu[i] mean_i over all walks, this rank running its share."""
    rank, size = world()
    local, count = _local(settings, rank, size)
    if count > 0:
        dV, dg, ds = native_scene.adjoint(P, local, adjoint, dLdu * (count / settings.nwalks))
    else:
        # no walks on this rank (nwalks < world size): contribute exact zeros
        # to the sum, without a launch whose inf/NaN walks would turn 0 * inf
        # into NaN on every rank
        dV, dg, ds = _zero_gradients(native_scene, adjoint, P.device)
    allreduce_sum_([dV, dg, ds])
    return dV, dg, ds


def _zero_gradients(native_scene, adjoint, device):
    """Zero dV (nV x dim), dg (nV) and dsrc (5) as the native adjoint returns
    them, None where the matching want_* flag is off."""
    nV, dim = int(native_scene.nV), int(native_scene.dim)
    f32 = torch.float32
    dV = torch.zeros((nV, dim), dtype=f32, device=device) if adjoint.want_dV else None
    dg = torch.zeros(nV, dtype=f32, device=device) if adjoint.want_dg else None
    ds = torch.zeros(5, dtype=f32, device=device) if adjoint.want_dsrc else None
    return dV, dg, ds
