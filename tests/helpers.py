"""Synthetic inputs shared by the tests and the benchmark (seeded NumPy)."""
from __future__ import annotations

import numpy as np


def ball_problem(n: int = 40, centre: float = 20.0, radius: float = 10.0, inside: float = 1.1):
    """Target J = `inside` in a ball of `radius` voxels around `centre`,
    1.0 elsewhere; the mask is the ball."""
    z, y, x = np.meshgrid(*[np.arange(n)] * 3, indexing="ij")
    m = (x - centre) ** 2 + (y - centre) ** 2 + (z - centre) ** 2 <= radius * radius
    return np.ascontiguousarray(np.where(m, inside, 1.0)), np.ascontiguousarray(m)


def masked_max(J, Jt, mask) -> float:
    d = np.abs(J - Jt)[mask]
    return float(d.max()) if d.size else 0.0
