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
