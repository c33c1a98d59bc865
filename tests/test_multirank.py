"""The multi-rank host path with world_size-2 gloo ranks on the CPU.

The GPU compute is replaced by a deterministic stand-in that has the same
contract as the native scene (per-walk values defined by (point, global walk
index)), so the test checks exactly what the sharding adds: walk ranges,
weights and the reductions.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


class FakeNative:
    """Per-walk value v(pt, wk) and gradient contributions, like the kernels:
    solve = mean over walks [offset, offset + nwalks); adjoint adds
    dLdu[pt] / nwalks * d v / d theta for each of those walks."""

    nV, dim = 5, 2

    @staticmethod
    def value(pt, wk):
        return np.sin(1.3 * pt + 0.7 * wk) + 0.1 * wk

    def solve(self, P, s):
        n = P.shape[0]
        w = np.arange(s.walk_offset, s.walk_offset + s.nwalks)
        v = np.array([[self.value(i, k) for k in w] for i in range(n)])
        return torch.tensor(v.mean(1), dtype=torch.float64)

    def adjoint(self, P, s, a, dLdu):
        n = P.shape[0]
        dV = torch.zeros(self.nV, self.dim, dtype=torch.float32) if a.want_dV else None
        dg = torch.zeros(self.nV, dtype=torch.float32) if a.want_dg else None
        ds = torch.zeros(5, dtype=torch.float32) if a.want_dsrc else None
        if s.nwalks < 1:
            raise AssertionError("the sharded adjoint must not launch a rank without walks")
        for i in range(n):
            for k in range(s.walk_offset, s.walk_offset + s.nwalks):
                W = float(dLdu[i]) / s.nwalks
                if dV is not None:
                    dV[(i + k) % self.nV] += W * torch.tensor([1.0, float(k)])
                if dg is not None:
                    dg[k % self.nV] += W
                if ds is not None:
                    ds[i % 5] += W * k
        return dV, dg, ds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, size, port, out, nwalks=11):
    sys.path.insert(0, str(ROOT / "diff-wos_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from wos import dist as wdist
    from wos.native import AdjointSettings, WalkSettings
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        P = torch.zeros(7, 2)
        s = WalkSettings(nwalks=nwalks, walk_offset=3, seed=1)
        fake = FakeNative()
        mean = wdist.sharded_solve(fake, P, s)
        dLdu = torch.linspace(-1.0, 2.0, 7)
        dV, dg, ds = wdist.sharded_adjoint(fake, P, s, AdjointSettings(want_dg=True, want_dsrc=True), dLdu)
        t = torch.tensor([float(rank + 1)])
        mx = wdist.max_over_ranks(3.0 * (rank + 1))
        out[rank] = (mean.numpy(), dV.numpy(), dg.numpy(), ds.numpy(), mx)
    finally:
        dist.destroy_process_group()


def test_shard_partition():
    from wos.dist import shard
    for n in (0, 1, 7, 64, 100):
        for size in (1, 2, 3, 8):
            parts = [shard(n, r, size) for r in range(size)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(size - 1))
            lens = [b - a for a, b in parts]
            assert max(lens) - min(lens) <= 1


@pytest.mark.timeout(120)
@pytest.mark.parametrize("nwalks", [11, 1])
def test_two_rank_gloo_matches_single_rank(nwalks):
    """nwalks = 1 leaves rank 1 without walks: it must add zeros, not launch."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out, nwalks)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    sys.path.insert(0, str(ROOT / "diff-wos_b200"))
    from wos.native import AdjointSettings, WalkSettings
    fake = FakeNative()
    P = torch.zeros(7, 2)
    s = WalkSettings(nwalks=nwalks, walk_offset=3, seed=1)
    ref_mean = fake.solve(P, s).numpy()
    ref = fake.adjoint(P, s, AdjointSettings(want_dg=True, want_dsrc=True), torch.linspace(-1.0, 2.0, 7))
    for r in range(2):
        mean, dV, dg, ds, mx = out[r]
        np.testing.assert_allclose(mean, ref_mean, rtol=1e-12)
        np.testing.assert_allclose(dV, ref[0].numpy(), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(dg, ref[1].numpy(), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(ds, ref[2].numpy(), rtol=1e-5, atol=1e-5)
        assert mx == 6.0
