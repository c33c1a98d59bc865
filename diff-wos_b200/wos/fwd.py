"""Common imports and helpers of the wos package (the reference's wos/fwd.py
re-exported Dr.Jit types; this build works on torch CUDA tensors)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

from .native import as_cuda, cuda_device

basedir = Path(__file__).resolve().parent.parent

EPSILON = 1e-3


def tensor(x, dtype=torch.float32) -> torch.Tensor:
    """CUDA tensor of dtype; torch inputs keep their autograd graph."""
    if isinstance(x, torch.Tensor):
        if x.device.type != "cuda":
            x = x.to(cuda_device())
        if x.dtype != dtype:
            x = x.to(dtype)
        return x
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=cuda_device())


def points(p, dim: int) -> torch.Tensor:
    """(n, dim) contiguous float32 CUDA points (detached)."""
    return as_cuda(p, torch.float32, dim).reshape(-1, dim)


__all__ = ["np", "torch", "basedir", "EPSILON", "tensor", "points"]
