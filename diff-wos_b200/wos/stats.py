"""Running statistics (reference: wos/stats.py:1-36)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Statistics:
    """Welford running mean / M2 / variance / 95% interval of a 1D stream."""

    def mean(self, x):
        x = np.asarray(x, np.float64)
        return np.cumsum(x) / (np.arange(len(x)) + 1)

    def m2(self, x):
        x = np.asarray(x, np.float64)
        mean = 0.0
        m2 = 0.0
        out = np.zeros(len(x))
        for i in range(len(x)):
            delta = x[i] - mean
            mean += delta / (i + 1)
            m2 += delta * (x[i] - mean)
            out[i] = m2
        return out

    def var(self, x):
        return self.m2(x) / (np.arange(len(x)) + 1)

    def ci(self, x):
        return 1.96 * np.sqrt(self.var(x) / np.sqrt(np.arange(len(x)) + 1))


def merge_solves(mean_a, var_a, n_a: int, mean_b, var_b, n_b: int):
    """Per-point mean and sample variance (n - 1 denominator, as the solve
    returns them) of two solves of the same points over disjoint walk
    ranges, by the pairwise update of Chan, Golub and LeVeque (1979).

    Walks are numbered: a solve with `walk_offset = k` runs walks k, k + 1,
    ... of every point, with the random numbers those walks have in any
    larger solve.  So a solve of n_a walks followed by one of n_b walks at
    walk_offset = n_a holds exactly the walks of one solve of n_a + n_b, and
    merging their (mean, var) gives that solve's estimate up to rounding: a
    long solve can stop after any call and resume with the next walk range.
    Works on numpy arrays and torch tensors alike; returns (mean, var)."""
    n = n_a + n_b
    if n_a <= 0 or n_b <= 0:
        return (mean_b, var_b) if n_a <= 0 else (mean_a, var_a)
    delta = mean_b - mean_a
    mean = mean_a + delta * (n_b / n)
    m2 = var_a * (n_a - 1) + var_b * (n_b - 1) + delta * delta * (n_a * n_b / n)
    return mean, m2 / (n - 1) if n > 1 else m2 * 0.0
