"""CPU restatement of the multi-resolution wrapper (test infrastructure).

This file is the checker of the device pyramid: only the tests, the smoke
check and the benchmark's CPU leg use it.  It restates
* the reference's ``displacement()`` driver (disptools/displacements.py:238-480),
* its ``redistribute_volume_change`` (``:224-229``),
* ``scale_image`` (disptools/drawing.py:23-69),
on NumPy arrays, with the C oracle (dt_oracle.c) solving each level.

Parity unpinned against the reference itself.  The reference smooths with
ITK's SmoothingRecursiveGaussian and resamples with ITK's
ResampleImageFilter, and SimpleITK is not installed here.  The filters below
are the ones the device kernels implement:
* the smoothing of 2.0 physical units as a recursive Gaussian, the method
  that SmoothingRecursiveGaussian is built on: R. Deriche, "Recursively
  implementing the Gaussian and its derivatives", INRIA research report
  1893 (1993), fourth-order causal + anticausal recursions with Deriche's
  published coefficients, normalised to unit DC gain, each recursion started
  in the steady state of the border value (a zero-flux border, as if the
  volume continued with its edge values); pinned by the filter's own
  properties (tests/test_pyramid_oracle.py), since ITK is absent;
* or, on request, a sampled Gaussian truncated at ceil(4 sigma) and
  normalised, with zero-flux borders;
* linear / nearest resampling over the same physical extent with ITK's
  half-voxel inside rule.
They are written operation for operation in the kernels' order, so the
device results can be checked bit for bit.  The driver's steps (padding,
redistribution, level sizes and spacings, mask reading, per-level it_max,
initial guess, crop) follow the reference's Python code line by line.
"""
from __future__ import annotations

import math

import numpy as np

from .oracle import Oracle


def gaussian_weights(sigma: float):
    """(radius, weights): exp(-k^2 / (2 sigma^2)) for |k| <= ceil(4 sigma),
    divided by their sum accumulated in increasing k."""
    if not sigma > 0.0:
        return 0, [1.0]
    r = math.ceil(4.0 * sigma)
    w = [math.exp(-(k * k) / (2.0 * sigma * sigma)) for k in range(-r, r + 1)]
    s = 0.0
    for v in w:
        s += v
    return r, [v / s for v in w]


def _smooth_axis(v: np.ndarray, axis: int, r: int, w) -> np.ndarray:
    n = v.shape[axis]
    acc = np.zeros(v.shape)
    for k in range(-r, r + 1):
        idx = np.clip(np.arange(n) + k, 0, n - 1)
        acc = acc + w[k + r] * np.take(v, idx, axis=axis)
    return acc


# Deriche's fourth-order approximation of the Gaussian (INRIA RR-1893, 1993):
# for x >= 0 and unit sigma,
#   g(x) ~ (a0 cos(w0 x) + a1 sin(w0 x)) exp(-b0 x) + (c0 cos(w1 x) + c1 sin(w1 x)) exp(-b1 x).
DERICHE_GAUSSIAN = (1.680, 3.735, 1.783, 0.6318, -0.6803, -0.2598, 1.723, 1.997)  # a0 a1 b0 w0 c0 c1 b1 w1


def deriche_coefficients(sigma: float):
    """(n, m, d, gc, ga) of the recursive Gaussian of `sigma` samples:
    causal y+[i] = sum_k n[k] x[i-k] - sum_k d[k] y+[i-1-k] (k = 0..3),
    anticausal y-[i] = sum_k m[k] x[i+1+k] - sum_k d[k] y-[i+1+k], y = y+ + y-;
    n and m scaled so the sum of the impulse response is 1; gc and ga the
    steady-state responses of the two recursions to a unit constant.  The
    numerators and denominator are the z-transforms of the causal part of
    g (two damped cosines) and of its mirror image."""
    a0, a1, b0, w0, c0, c1, b1, w1 = DERICHE_GAUSSIAN
    eb0, eb1 = math.exp(-b0 / sigma), math.exp(-b1 / sigma)
    cw0, sw0 = math.cos(w0 / sigma), math.sin(w0 / sigma)
    cw1, sw1 = math.cos(w1 / sigma), math.sin(w1 / sigma)
    n0 = a0 + c0
    n1 = eb1 * (c1 * sw1 - (c0 + 2.0 * a0) * cw1) + eb0 * (a1 * sw0 - (2.0 * c0 + a0) * cw0)
    n2 = (2.0 * eb0 * eb1 * ((a0 + c0) * cw1 * cw0 - a1 * cw1 * sw0 - c1 * cw0 * sw1)
          + c0 * eb0 * eb0 + a0 * eb1 * eb1)
    n3 = eb1 * eb0 * eb0 * (c1 * sw1 - c0 * cw1) + eb0 * eb1 * eb1 * (a1 * sw0 - a0 * cw0)
    d1 = -2.0 * eb1 * cw1 - 2.0 * eb0 * cw0
    d2 = 4.0 * cw1 * cw0 * eb0 * eb1 + eb1 * eb1 + eb0 * eb0
    d3 = -2.0 * cw0 * eb0 * eb1 * eb1 - 2.0 * cw1 * eb1 * eb0 * eb0
    d4 = eb0 * eb0 * eb1 * eb1
    m1, m2, m3, m4 = n1 - d1 * n0, n2 - d2 * n0, n3 - d3 * n0, -d4 * n0
    den = 1.0 + d1 + d2 + d3 + d4
    gain = (n0 + n1 + n2 + n3 + m1 + m2 + m3 + m4) / den
    n = [n0 / gain, n1 / gain, n2 / gain, n3 / gain]
    m = [m1 / gain, m2 / gain, m3 / gain, m4 / gain]
    gc = (n[0] + n[1] + n[2] + n[3]) / den
    ga = (m[0] + m[1] + m[2] + m[3]) / den
    return n, m, [d1, d2, d3, d4], gc, ga


def _recursive_axis(v: np.ndarray, axis: int, sigma: float, t) -> np.ndarray:
    """One axis of the recursive Gaussian over every line of `v` (float64),
    result rounded to `t`.  The anticausal pass runs first and is stored in
    `t`; the causal pass adds itself to it.  Every sum is formed left to
    right, each operation rounded, as in the kernel."""
    if not sigma > 0.0:
        return v.astype(t)
    n, m, d, gc, ga = deriche_coefficients(sigma)
    x = np.moveaxis(v, axis, 0)
    L = x.shape[0]
    ym = np.empty(x.shape, dtype=t)
    xe = x[L - 1]
    xn = [xe, xe, xe, xe]                       # x[i+1 .. i+4]
    yn = [xe * ga, xe * ga, xe * ga, xe * ga]   # y-[i+1 .. i+4]
    for i in range(L - 1, -1, -1):
        acc = m[0] * xn[0]
        acc = acc + m[1] * xn[1]
        acc = acc + m[2] * xn[2]
        acc = acc + m[3] * xn[3]
        acc = acc - d[0] * yn[0]
        acc = acc - d[1] * yn[1]
        acc = acc - d[2] * yn[2]
        acc = acc - d[3] * yn[3]
        ym[i] = acc
        xn = [x[i], xn[0], xn[1], xn[2]]
        yn = [acc, yn[0], yn[1], yn[2]]
    out = np.empty(x.shape, dtype=t)
    x0 = x[0]
    xp = [x0, x0, x0]                           # x[i-1 .. i-3]
    yp = [x0 * gc, x0 * gc, x0 * gc, x0 * gc]   # y+[i-1 .. i-4]
    for i in range(L):
        acc = n[0] * x[i]
        acc = acc + n[1] * xp[0]
        acc = acc + n[2] * xp[1]
        acc = acc + n[3] * xp[2]
        acc = acc - d[0] * yp[0]
        acc = acc - d[1] * yp[1]
        acc = acc - d[2] * yp[2]
        acc = acc - d[3] * yp[3]
        out[i] = acc + ym[i].astype(np.float64)
        xp = [x[i], xp[0], xp[1]]
        yp = [acc, yp[0], yp[1], yp[2]]
    return np.moveaxis(out, 0, axis)


def smooth(vol: np.ndarray, sigma_xyz, method: str = "recursive") -> np.ndarray:
    """Separable Gaussian of a [C, nz, ny, nx] array (x, then y, then z);
    each pass computes in float64 and rounds to the array's type.
    ``method`` "recursive" (Deriche, the default) or "sampled"."""
    t = vol.dtype
    v = vol
    for axis, sigma in zip((3, 2, 1), sigma_xyz):
        if method == "recursive":
            v = _recursive_axis(v.astype(np.float64), axis, float(sigma), t)
        elif method == "sampled":
            r, w = gaussian_weights(float(sigma))
            v = _smooth_axis(v.astype(np.float64), axis, r, w).astype(t)
        else:
            raise ValueError(f"unknown smoothing method {method!r}")
    return v


def _coords(n: int, n2: int):
    p = (np.arange(n2, dtype=np.float64) * n) / n2
    inside = (p >= -0.5) & (p < n - 0.5)
    return p, inside


def resample(vol: np.ndarray, size_zyx, nearest: bool = False) -> np.ndarray:
    """Resampling of a [C, nz, ny, nx] array onto size_zyx voxels over the
    same physical extent (continuous index i * n / n2; 0 outside
    [-0.5, n - 0.5); linear along x, then y, then z, or nearest)."""
    t = vol.dtype
    v = vol.astype(np.float64)
    _, nz, ny, nx = v.shape
    nz2, ny2, nx2 = (int(s) for s in size_zyx)
    pz, iz = _coords(nz, nz2)
    py, iy = _coords(ny, ny2)
    px, ix = _coords(nx, nx2)
    inside = iz[:, None, None] & iy[None, :, None] & ix[None, None, :]
    if nearest:
        zi = np.minimum(np.floor(pz + 0.5).astype(np.int64), nz - 1).clip(0)
        yi = np.minimum(np.floor(py + 0.5).astype(np.int64), ny - 1).clip(0)
        xi = np.minimum(np.floor(px + 0.5).astype(np.int64), nx - 1).clip(0)
        out = v[:, zi][:, :, yi][:, :, :, xi]
    else:
        def split(p, n):
            f0 = np.floor(p)
            frac = p - f0
            i0 = np.maximum(f0.astype(np.int64), 0)
            i1 = np.minimum(f0.astype(np.int64) + 1, n - 1)
            return i0, i1, frac

        z0, z1, fz = split(pz, nz)
        y0, y1, fy = split(py, ny)
        x0, x1, fx = split(px, nx)

        def lerp(a, b, f):
            return a + (b - a) * f

        def plane(zi, yi):
            g = v[:, zi][:, :, yi]
            return lerp(g[..., x0], g[..., x1], fx[None, None, None, :])

        c00, c10 = plane(z0, y0), plane(z0, y1)
        c01, c11 = plane(z1, y0), plane(z1, y1)
        fyb = fy[None, None, :, None]
        c0 = lerp(c00, c10, fyb)
        c1 = lerp(c01, c11, fyb)
        out = lerp(c0, c1, fz[None, :, None, None])
    out = np.where(inside[None], out, 0.0)
    return out.astype(t)


def scale_image(vol: np.ndarray, spacing_xyz, size_zyx, nearest: bool = False,
                method: str = "recursive") -> np.ndarray:
    """disptools/drawing.py:23-69: smooth by 2.0 physical units, resample."""
    sig = [2.0 / float(s) for s in spacing_xyz]
    return resample(smooth(vol, sig, method), size_zyx, nearest)


def displacement(jacobian, *, levels=1, pad=0, redistribute=False, mask=None, initial_guess=None,
                 spacing=(1.0, 1.0, 1.0), it_max=50000, algorithm="gradient", field_dtype=np.float64,
                 smoothing="recursive", solver=None, **params):
    """disptools/displacements.py:238-480 on NumPy arrays, each level solved
    by the C oracle (or by ``solver``, an object with the oracle's ``solve``,
    such as the reference library).  ``field_dtype`` float32 rounds the
    fields passed between levels like the mixed-precision device path."""
    o = solver if solver is not None else Oracle(4)
    J = np.array(jacobian, dtype=np.float64)
    m = np.ones(J.shape) if mask is None else np.asarray(mask, dtype=np.float64)
    its = list(it_max) if isinstance(it_max, (list, tuple)) else [it_max] * levels
    p = pad + 1 if pad > 0 else 1                                   # :443-450
    if redistribute:                                                 # :224-229
        correction = -(np.sum(J) - J.size) / (J.size - np.count_nonzero(m))
        J[m == 0.0] += correction
    m = np.pad(m, p, mode="constant", constant_values=0.0)           # :455
    J = np.pad(J, p, mode="edge")                                    # :456
    sizes = [J.shape]                                                # :459-463
    for _ in range(1, levels):
        sizes.append(tuple(s // 2 for s in sizes[-1]))
    n0 = J.shape[::-1]
    spacings = [tuple(float(sp) * n / k for sp, n, k in zip(spacing, n0, sz[::-1])) for sz in sizes]
    Js = [J] + [scale_image(J[None], spacings[0], sizes[i], method=smoothing)[0] for i in range(1, levels)]
    ms = [m] + [scale_image(m[None], spacings[0], sizes[i], nearest=True, method=smoothing)[0]
                for i in range(1, levels)]
    field = None if initial_guess is None else np.asarray(initial_guess, dtype=field_dtype)
    field_spacing = spacing
    for lv, it in zip(range(levels - 1, -1, -1), its):              # :476-480
        if field is not None:
            field = scale_image(field.astype(field_dtype), field_spacing, sizes[lv], method=smoothing)
        f0 = None if field is None else field.astype(np.float64)
        out = o.solve(algorithm, np.ascontiguousarray(Js[lv]), np.ascontiguousarray(ms[lv] != 0),
                      field=f0, spacing=spacings[lv], it_max=it, **params)
        out = out[0] if isinstance(out, tuple) else out  # the oracle also returns its statistics
        field = out.astype(field_dtype)
        field_spacing = spacings[lv]
    return field[:, p:-p, p:-p, p:-p].astype(np.float64)             # :483
