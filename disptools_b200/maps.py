"""Jacobian-map utilities on the device.

Mirror of the reference's map functions (disptools/displacements.py:486-668)
on arrays instead of SimpleITK images:

* :func:`jacobian_to_volume_change` (``:628-668``);
* :func:`average_jacobian` (``:571-625``): geometric mean of Jacobian maps,
  each thresholded to [epsilon, 1e9] (outside values become epsilon);
* :func:`average_jacobian_from_displacements` (``:486-568``): geometric mean
  of the Jacobians of displacement fields, each regularised (values below
  epsilon become epsilon).

The arithmetic runs in this package's kernels (``dt_maps.cu``); the logs are
accumulated in FP64 and the mean is ``exp((1 / n) * sum)``, as in the
reference.  Maps and fields may be NumPy arrays, device tensors or file
names (a glob pattern, as in the reference): ``.vtk`` through
:mod:`disptools_b200.io`, ``.rvf`` for fields, ``.npy`` arrays.
"""
from __future__ import annotations

import glob as _glob
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _native as N
from . import io as fio
from . import torch_ops

# Clamp modes of dtb_log_jacobian_accumulate_device
CLAMP_THRESHOLD = 0   # values outside [epsilon, 1e9] become epsilon
CLAMP_REGULARISE = 1  # values below epsilon become epsilon


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _prec(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return N.precision_code("fp64")
    if t.dtype == torch.float32:
        return N.precision_code("mixed")
    raise TypeError("maps must be float32 or float64")


def _device_tensor(a, device=None) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.contiguous() if a.is_cuda else a.to(device or "cuda").contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device or "cuda")


def jacobian_to_volume_change(jacobian, epsilon: float = 1e-5):
    """Volume-change map: J - 1 where J >= 1, 1 - 1/J where J < 1, with J
    below epsilon replaced by epsilon.  NumPy in, NumPy out; a device tensor
    gives a device tensor of its dtype (float32 or float64)."""
    host = not isinstance(jacobian, torch.Tensor)
    J = _device_tensor(jacobian)
    out = torch.empty_like(J)
    with torch.cuda.device(J.device):
        N.check(N.lib.dtb_volume_change_device(_prec(J), J.numel(), float(epsilon), J.data_ptr(),
                                               out.data_ptr(), _stream(J)))
    return out.cpu().numpy() if host else out


def _expand(items) -> list:
    if isinstance(items, str):
        return list(_glob.glob(items))
    return list(items)


def _load_map(item):
    if isinstance(item, str):
        if item.endswith(".npy"):
            return np.load(item), None
        data, sp = fio.read_vtk(item)
        if data.shape[0] != 1:
            raise ValueError(f"{item}: expected a scalar map")
        return data[0], sp
    return item, None


def _load_field(item, spacing):
    if isinstance(item, str):
        if item.endswith(".rvf"):
            return fio.read_rvf(item)
        if item.endswith(".npy"):
            return np.load(item), spacing
        return fio.read_vtk(item)
    return item, spacing


def _geometric_mean(maps: list, mode: int, epsilon: float):
    if not maps:
        raise ValueError("no maps")
    acc = None
    host = True
    for J in maps:
        host &= not isinstance(J, torch.Tensor)
        Jd = _device_tensor(J)
        if acc is None:
            acc = torch.zeros(Jd.shape, dtype=torch.float64, device=Jd.device)
        elif Jd.shape != acc.shape:
            raise ValueError("all maps must have the same shape")
        with torch.cuda.device(Jd.device):
            N.check(N.lib.dtb_log_jacobian_accumulate_device(_prec(Jd), mode, Jd.numel(), float(epsilon),
                                                             Jd.data_ptr(), acc.data_ptr(), _stream(Jd)))
    out = torch.empty_like(acc)
    with torch.cuda.device(acc.device):
        N.check(N.lib.dtb_exp_mean_device(N.precision_code("fp64"), acc.numel(), 1.0 / len(maps),
                                          acc.data_ptr(), out.data_ptr(), _stream(acc)))
    return out.cpu().numpy() if host else out


def average_jacobian(maps, epsilon: float = 1e-5):
    """Geometric mean of Jacobian maps (arrays, tensors, or a glob pattern of
    ``.vtk`` / ``.npy`` files), each thresholded to [epsilon, 1e9]."""
    items = [_load_map(m)[0] for m in _expand(maps)]
    return _geometric_mean(items, CLAMP_THRESHOLD, epsilon)


def average_jacobian_from_displacements(fields, epsilon: float = 1e-5,
                                        spacing: Sequence[float] = (1.0, 1.0, 1.0)):
    """Geometric mean of the Jacobians of displacement fields (``[3, nz, ny,
    nx]`` arrays or tensors, or a glob pattern of ``.rvf`` / ``.vtk`` /
    ``.npy`` files; files carry their own spacing, arrays use
    ``spacing``), each regularised at epsilon.  The Jacobians are computed
    in FP64 with the reference stencil."""
    items = _expand(fields)
    Js = []
    for item in items:
        f, sp = _load_field(item, spacing)
        fd = _device_tensor(f).to(torch.float64).contiguous()
        Js.append(torch_ops.jacobian_raw(fd, sp))
    host = not any(isinstance(f, torch.Tensor) for f in items)
    out = _geometric_mean(Js, CLAMP_REGULARISE, epsilon)
    return out.cpu().numpy() if host else out
