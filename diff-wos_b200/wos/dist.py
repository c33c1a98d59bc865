"""Multi-GPU helpers: one process per GPU, torch.distributed for plumbing.

Query points x walks are independent, so a solve shards by contiguous point
ranges with the scene (and its LBVH) replicated on every rank; the forward
needs no exchange, the adjoint one sum-all-reduce of the gradient buffers
(per-vertex dV, dg and the 5 source coefficients).
"""
from __future__ import annotations

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
    """In-place sum over ranks of every non-None tensor (one flat buffer)."""
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


def sharded_adjoint(native_scene, P, settings, adjoint, dLdu):
    """Adjoint over all points with this rank computing its shard; the
    gradient buffers are summed across ranks.  Walk indices keep their global
    point index, so results equal a single-GPU run up to summation order."""
    rank, size = world()
    n = P.shape[0]
    a, b = shard(n, rank, size)
    dV, dg, ds = native_scene.adjoint_range(P, settings, adjoint, dLdu, a, b)
    allreduce_sum_([dV, dg, ds])
    return dV, dg, ds
