"""Seeded synthetic target maps and fields (NumPy / SciPy).

These stand in for data sets (the reference publishes no benchmark data):

* :func:`blob_problem` — target J = clip(exp(sum of isotropic Gaussian
  blobs), 0.7, 1.4), mask = voxels with |log J| > 0.01 dilated by 3
  (:func:`blob_problem_device` computes it with torch on a device);
* :func:`ellipsoid_problem` — 1 to 4 ellipsoids of J in [0.80, 0.95],
  J = 1 elsewhere, mask = ellipsoids dilated by 2;
* :func:`smooth_field` — Gaussian-filtered white noise scaled to a maximum
  displacement.

Arrays are in the library layout: maps ``[nz, ny, nx]`` float64, masks bool,
fields ``[3, nz, ny, nx]`` float64.
"""
from __future__ import annotations

import numpy as np


def _dilate(mask: np.ndarray, radius: float) -> np.ndarray:
    """Binary dilation by a Euclidean ball of `radius` voxels."""
    from scipy.ndimage import distance_transform_edt
    if not mask.any():
        return mask.copy()
    return distance_transform_edt(~mask) <= radius


def blob_problem(shape=(256, 256, 256), blobs: int = 16, seed: int = 0,
                 sigma=(8.0, 24.0), amplitude: float = 0.25):
    """log J = sum_b A_b exp(-|x - c_b|^2 / (2 sigma_b^2)), centres uniform in
    the grid, sigma_b ~ U(sigma), A_b ~ U(-amplitude, amplitude); J clipped to
    [0.7, 1.4]; mask = |log J| > 0.01 dilated by 3."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    logj = np.zeros(shape)
    z = np.arange(nz, dtype=np.float64)
    y = np.arange(ny, dtype=np.float64)
    x = np.arange(nx, dtype=np.float64)
    for _ in range(blobs):
        c = rng.uniform([0, 0, 0], [nz, ny, nx])
        s = rng.uniform(*sigma)
        a = rng.uniform(-amplitude, amplitude)
        ez = np.exp(-(z - c[0]) ** 2 / (2 * s * s))
        ey = np.exp(-(y - c[1]) ** 2 / (2 * s * s))
        ex = np.exp(-(x - c[2]) ** 2 / (2 * s * s))
        logj += a * ez[:, None, None] * (ey[:, None] * ex[None, :])[None]
    J = np.clip(np.exp(logj), 0.7, 1.4)
    mask = _dilate(np.abs(logj) > 0.01, 3.0)
    return np.ascontiguousarray(J), np.ascontiguousarray(mask)


def blob_problem_device(shape=(256, 256, 256), blobs: int = 16, seed: int = 0,
                        sigma=(8.0, 24.0), amplitude: float = 0.25, device="cuda"):
    """:func:`blob_problem` computed with torch on `device` (float64), for
    volumes where the NumPy version is slow: the same random draws, the
    same formulas, the dilation by 3 as a union of the mask shifted by every
    integer offset of length <= 3 (which is what a Euclidean distance <= 3
    to the mask means on the grid).  Returns (J float64, mask bool) tensors;
    exp() may round differently from NumPy's in the last bit."""
    import torch
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    dev = torch.device(device)
    z = torch.arange(nz, dtype=torch.float64, device=dev)
    y = torch.arange(ny, dtype=torch.float64, device=dev)
    x = torch.arange(nx, dtype=torch.float64, device=dev)
    logj = torch.zeros(shape, dtype=torch.float64, device=dev)
    for _ in range(blobs):
        c = rng.uniform([0, 0, 0], [nz, ny, nx])
        s = rng.uniform(*sigma)
        a = rng.uniform(-amplitude, amplitude)
        ez = torch.exp(-(z - c[0]) ** 2 / (2 * s * s))
        ey = torch.exp(-(y - c[1]) ** 2 / (2 * s * s))
        ex = torch.exp(-(x - c[2]) ** 2 / (2 * s * s))
        logj += a * ez[:, None, None] * (ey[:, None] * ex[None, :])[None]
    J = torch.clamp(torch.exp(logj), 0.7, 1.4)
    core = logj.abs() > 0.01
    mask = core.clone()
    r = 3
    for dz in range(-r, r + 1):
        for dy in range(-r, r + 1):
            for dx in range(-r, r + 1):
                if (dz, dy, dx) == (0, 0, 0) or dz * dz + dy * dy + dx * dx > r * r:
                    continue
                dst = tuple(slice(max(d, 0), n + min(d, 0)) for d, n in zip((dz, dy, dx), shape))
                src = tuple(slice(max(-d, 0), n + min(-d, 0)) for d, n in zip((dz, dy, dx), shape))
                mask[dst] |= core[src]
    return J, mask


def ellipsoid_problem(shape, seed: int = 0, count=None):
    """1-4 random ellipsoids (semi-axes U(4, 20) voxels) of J ~ U(0.80, 0.95);
    J = 1 elsewhere; mask = the ellipsoids dilated by 2.

    Each ellipsoid is evaluated and dilated inside its bounding box grown by
    3 voxels: a dilation of a union is the union of the dilations, and no
    voxel farther than 2 from an ellipsoid joins the mask."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    J = np.ones(shape)
    mask = np.zeros(shape, bool)
    for _ in range(int(count or rng.integers(1, 5))):
        r = rng.uniform(4, 20, 3)
        c = rng.uniform([0, 0, 0], [nz, ny, nx])
        v = rng.uniform(0.80, 0.95)
        lo = [max(0, int(np.floor(c[a] - r[a])) - 3) for a in range(3)]
        hi = [min(shape[a], int(np.ceil(c[a] + r[a])) + 4) for a in range(3)]
        z = np.arange(lo[0], hi[0])[:, None, None]
        y = np.arange(lo[1], hi[1])[None, :, None]
        x = np.arange(lo[2], hi[2])[None, None, :]
        e = ((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2 <= 1
        box = tuple(slice(a, b) for a, b in zip(lo, hi))
        J[box][e] = v
        mask[box] |= _dilate(e, 2.0)
    return np.ascontiguousarray(J), np.ascontiguousarray(mask)


def batch_sizes(count: int = 64, low: int = 48, high: int = 192, seed: int = 0):
    """Per-axis sizes drawn uniformly from [low, high]."""
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.integers(low, high + 1, 3)) for _ in range(count)]


def smooth_field(shape, sigma: float = 6.0, max_disp: float = 3.0, seed: int = 0) -> np.ndarray:
    """White noise N(0, 1) filtered by a Gaussian of `sigma` voxels and scaled
    so that max |u| = max_disp; shape ``[3, *shape]``."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    f = np.empty((3,) + tuple(shape))
    for c in range(3):
        f[c] = gaussian_filter(rng.standard_normal(shape), sigma, mode="wrap")
    f *= max_disp / np.max(np.abs(f))
    return np.ascontiguousarray(f)
