"""Multi-resolution displacement generation on the device.

Mirror of the reference's Python wrapper ``displacement()``
(disptools/displacements.py:238-480) on NumPy arrays instead of SimpleITK
images.  The steps follow the reference's code, in its order:

1. The padding is ``pad + 1`` voxels on every side, at least 1 (``:443-450``).
   The target Jacobian is padded zero-flux (edge values repeated) and the
   mask with zeros (``:455-456``).
2. With ``redistribute``, the volume change is redistributed before padding:
   every voxel outside the mask gets ``-(sum J - N) / (N - count(mask))``
   added (``redistribute_volume_change``, ``:224-229``).
3. Level ``i`` has ``size_{i-1} // 2`` voxels per axis.  Every level is
   scaled from the full-resolution padded images (``:459-463``): the target
   Jacobian with linear interpolation, the mask with nearest neighbour.  In
   both cases the image is first smoothed by 2.0 physical units, as
   ``scale_image`` does for every interpolator (disptools/drawing.py:23-69).
   A voxel belongs to a level's mask where the sampled value is non-zero,
   which is how ``_displacement`` reads masks (``astype(bool)``).
4. Level spacing is ``s * n / n_i`` per axis, so the physical extent is
   preserved.
5. ``it_max`` is one value for every level or one per level, coarsest first
   (``:466-470``).
6. The levels are solved from the coarsest up (``:476-480``).  Each level
   starts from the previous level's field, scaled to its size by the same
   ``scale_image``.  A given ``initial_guess`` goes through it as well, at
   the coarsest level.
7. The padding is cropped from the finest field (``:483``).

Smoothing and resampling run as this package's CUDA kernels
(``dtb_smooth_recursive_device``, ``dtb_resample_device``), and every level
is solved by the device solver on device-resident tensors.  Padding and
redistribution are one-off steps, in NumPy for NumPy inputs and in torch for
device tensors.  The reference's filters are ITK's recursive Gaussian and
ResampleImageFilter.  The smoothing kernel implements the same method,
Deriche's recursive Gaussian (INRIA RR-1893, 1993), from its publication;
``smoothing="sampled"`` selects a truncated sampled Gaussian
(``dtb_smooth_device``) instead.  The resampling kernel restates the
resampler's interpolation rules (see ``include/disptools_b200.h``).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from . import _native as N
from . import torch_ops

SMOOTH_SIGMA = 2.0  # physical units, disptools/drawing.py:65


def _prec(t: torch.Tensor) -> int:
    return N.precision_code("fp64" if t.dtype == torch.float64 else "mixed")


SMOOTHING = ("recursive", "sampled")


def smooth(vol: torch.Tensor, sigma_vox: Sequence[float], method: str = "recursive") -> torch.Tensor:
    """Gaussian smoothing of a ``[C, nz, ny, nx]`` (or ``[nz, ny, nx]``)
    device tensor; ``sigma_vox`` = (sigma_x, sigma_y, sigma_z) in voxels.
    ``method``: "recursive" (Deriche's recursive Gaussian, the filter behind
    the reference's sitk.SmoothingRecursiveGaussian; the default) or
    "sampled" (a truncated sampled Gaussian)."""
    if method not in SMOOTHING:
        raise ValueError(f"smoothing method must be one of {SMOOTHING}, got {method!r}")
    fn = N.lib.dtb_smooth_recursive_device if method == "recursive" else N.lib.dtb_smooth_device
    v = vol if vol.dim() == 4 else vol.unsqueeze(0)
    v = v.contiguous()
    out = torch.empty_like(v)
    scratch = torch.empty_like(v)
    c, nz, ny, nx = v.shape
    with torch.cuda.device(v.device):
        N.check(fn(_prec(v), c, nx, ny, nz, *map(float, sigma_vox), v.data_ptr(), out.data_ptr(),
                   scratch.data_ptr(), torch.cuda.current_stream(v.device).cuda_stream))
    return out if vol.dim() == 4 else out[0]


def resample(vol: torch.Tensor, size_zyx: Sequence[int], nearest: bool = False) -> torch.Tensor:
    """Resampling of a ``[C, nz, ny, nx]`` (or ``[nz, ny, nx]``) device tensor
    onto ``size_zyx`` voxels spanning the same physical extent."""
    v = vol if vol.dim() == 4 else vol.unsqueeze(0)
    v = v.contiguous()
    c, nz, ny, nx = v.shape
    nz2, ny2, nx2 = (int(s) for s in size_zyx)
    out = torch.empty((c, nz2, ny2, nx2), dtype=v.dtype, device=v.device)
    with torch.cuda.device(v.device):
        N.check(N.lib.dtb_resample_device(_prec(v), 1 if nearest else 0, c, nx, ny, nz, nx2, ny2, nz2,
                                          v.data_ptr(), out.data_ptr(),
                                          torch.cuda.current_stream(v.device).cuda_stream))
    return out if vol.dim() == 4 else out[0]


def scale_image(vol: torch.Tensor, spacing_xyz: Sequence[float], size_zyx: Sequence[int],
                nearest: bool = False, method: str = "recursive") -> torch.Tensor:
    """scale_image (disptools/drawing.py:23-69): smooth by 2.0 physical units,
    then resample onto ``size_zyx`` voxels over the same extent."""
    sig = [SMOOTH_SIGMA / float(s) for s in spacing_xyz]
    return resample(smooth(vol, sig, method), size_zyx, nearest)


def level_geometry(shape_zyx: Sequence[int], spacing_xyz: Sequence[float], levels: int):
    """Sizes ``[nz, ny, nx]`` and spacings ``(dx, dy, dz)`` of the pyramid,
    finest first: each level halves the previous size (integer division) and
    keeps the physical extent of the finest level."""
    sizes = [tuple(int(s) for s in shape_zyx)]
    for _ in range(1, levels):
        sizes.append(tuple(s // 2 for s in sizes[-1]))
    n0 = sizes[0][::-1]  # x, y, z
    spacings = [tuple(float(sp) * n / m for sp, n, m in zip(spacing_xyz, n0, sz[::-1])) for sz in sizes]
    return sizes, spacings


def displacement(jacobian, *, levels: int = 1, pad: int = 0, redistribute: bool = False, mask=None,
                 initial_guess=None, spacing: Sequence[float] = (1.0, 1.0, 1.0),
                 epsilon: float = 9.99e-4, tolerance: float = 0.2, it_max=50000, alpha: float = 1.2,
                 beta: float = 0.5, gamma: float = 0.1, delta: float = 1e-3, zeta: float = 10.0,
                 theta: float = 1e-6, iota: float = 1e-9, strict: bool = False, eta: float = 0.1,
                 eta_max: float = 0.4, algorithm: str = "gradient", precision: str = "mixed",
                 device=None, return_stats: bool = False, smoothing: str = "recursive"):
    """Displacement field ``[3, nz, ny, nx]`` whose Jacobian matches
    ``jacobian`` (``[nz, ny, nx]``) in ``mask``, through a ``levels``-level
    pyramid (see the module docstring for the steps).  NumPy inputs give a
    float64 NumPy result; a device tensor ``jacobian`` keeps the whole
    computation on its device and gives a device tensor of the solver's
    element type.
    ``spacing`` is (dx, dy, dz).  ``precision`` selects the device solver
    (``"mixed"``: FP32 fields, ``"fp64"``); the target and mask pyramids are
    built in FP64.  ``algorithm`` is "gradient", "greedy" or "matching"; the
    matching solver always keeps float64 fields (it computes in FP32).  With ``return_stats`` also returns the per-level solver
    statistics, coarsest first.  ``smoothing`` is the anti-aliasing filter
    of every scaling: "recursive" (the default) or "sampled"."""
    if smoothing not in SMOOTHING:
        raise ValueError(f"smoothing must be one of {SMOOTHING}")
    if levels < 1:
        raise ValueError("levels must be at least 1")
    if algorithm not in ("gradient", "greedy", "matching"):
        raise ValueError("algorithm must be 'gradient', 'greedy' or 'matching'")
    if precision not in ("mixed", "fp64"):
        raise ValueError("precision must be 'mixed' or 'fp64'")
    if isinstance(it_max, (list, tuple)):
        if len(it_max) != levels:
            raise ValueError("len(it_max) should equal the value of `levels`")
        its = [int(v) for v in it_max]
    else:
        its = [int(it_max)] * levels
    p = pad + 1 if pad > 0 else 1
    if len(tuple(jacobian.shape)) == 3:
        # Every level must keep 3 voxels per axis (the solver's minimum):
        # checked before any work on the device.
        sizes0, _ = level_geometry(tuple(int(s) + 2 * p for s in jacobian.shape), spacing, levels)
        if min(sizes0[-1]) < 3:
            raise ValueError(f"level {levels - 1} would be {sizes0[-1]} voxels, below 3 along an axis: "
                             "use fewer levels")
    on_device = isinstance(jacobian, torch.Tensor)
    if on_device:
        # Device tensors stay on their device: padding and redistribution in
        # torch (the redistribution's sum may round differently from NumPy's).
        dev = jacobian.device
        J0 = jacobian.to(torch.float64)
        if J0.dim() != 3:
            raise ValueError("jacobian must be [nz, ny, nx]")
        m0 = torch.ones_like(J0) if mask is None else torch.as_tensor(mask, device=dev).to(torch.float64)
        if m0.shape != J0.shape:
            raise ValueError("the shapes of the Jacobian and the mask must agree")
        if redistribute:
            J0 = J0.clone()
            correction = -(J0.sum() - J0.numel()) / (J0.numel() - torch.count_nonzero(m0))
            J0[m0 == 0.0] += correction
        m0 = torch.nn.functional.pad(m0[None, None], (p,) * 6, mode="constant", value=0.0)[0, 0]
        J0 = torch.nn.functional.pad(J0[None, None], (p,) * 6, mode="replicate")[0, 0]
        shape0 = tuple(J0.shape)
    else:
        J = np.array(jacobian, dtype=np.float64)
        if J.ndim != 3:
            raise ValueError("jacobian must be [nz, ny, nx]")
        m = np.ones(J.shape) if mask is None else np.asarray(mask, dtype=np.float64)
        if m.shape != J.shape:
            raise ValueError("the shapes of the Jacobian and the mask must agree")
        if redistribute:
            correction = -(np.sum(J) - J.size) / (J.size - np.count_nonzero(m))
            J[m == 0.0] += correction
        m = np.pad(m, p, mode="constant", constant_values=0.0)
        J = np.pad(J, p, mode="edge")
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        J0 = torch.from_numpy(J).to(dev)
        m0 = torch.from_numpy(m).to(dev)
        shape0 = J.shape

    # The matching solver takes float64 arrays (it computes in FP32 inside).
    ftype = torch.float64 if precision == "fp64" or algorithm == "matching" else torch.float32
    sizes, spacings = level_geometry(shape0, spacing, levels)
    # Every coarser level is scaled from the same full-resolution images with
    # the same smoothing (2.0 physical units at the finest spacing), so each
    # image is smoothed once and then resampled per level: scale_image's
    # result for every level, with one smoothing pass instead of one a level.
    Js, ms = [J0], [m0]
    if levels > 1:
        sig0 = [SMOOTH_SIGMA / float(s) for s in spacings[0]]
        sJ0, sm0 = smooth(J0, sig0, smoothing), smooth(m0, sig0, smoothing)
        Js += [resample(sJ0, sizes[i]) for i in range(1, levels)]
        ms += [resample(sm0, sizes[i], nearest=True) for i in range(1, levels)]
        del sJ0, sm0

    field = None
    field_spacing = spacing
    if initial_guess is not None:
        g = (initial_guess if isinstance(initial_guess, torch.Tensor)
             else torch.from_numpy(np.ascontiguousarray(initial_guess, dtype=np.float64)))
        if tuple(g.shape) != (3,) + tuple(jacobian.shape):
            raise ValueError("initial_guess must be [3, nz, ny, nx] like the Jacobian")
        field = g.to(dev, ftype).contiguous()
    params = dict(epsilon=epsilon, tolerance=tolerance, eta=eta, eta_max=eta_max, alpha=alpha,
                  beta=beta, gamma=gamma, delta=delta, zeta=zeta, theta=theta, iota=iota,
                  strict=strict)
    stats = []
    for lv, it in zip(range(levels - 1, -1, -1), its):
        size, sp = sizes[lv], spacings[lv]
        if field is not None:
            field = scale_image(field, field_spacing, size, method=smoothing)
        else:
            field = torch.zeros((3,) + size, dtype=ftype, device=dev)
        Jl = Js[lv].to(ftype).contiguous()
        ml = (ms[lv] != 0).contiguous()
        st = torch_ops.solve(Jl, ml, field, spacing=sp, algorithm=algorithm, it_max=it, **params)
        stats.append(st)
        field_spacing = sp
    out = field[:, p:-p, p:-p, p:-p]
    out = out.contiguous() if on_device else out.to(torch.float64).cpu().numpy()
    return (out, stats) if return_stats else out
