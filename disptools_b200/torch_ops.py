"""Device-tensor entry points and the differentiable Jacobian.

PyTorch supplies device memory and the current stream; every computation is a
kernel of ``libdisptools_b200.so`` called through the C ABI with raw device
pointers.  Tensors must be CUDA, C-contiguous, float32 (mixed path) or
float64 (FP64 path); fields are ``[3, nz, ny, nx]`` (or a leading batch
dimension for :func:`jacobian`), scalar maps ``[nz, ny, nx]``.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import torch

from . import _native as N
from .api import make_params


def _precision(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return N.PRECISION_MIXED
    if t.dtype == torch.float64:
        return N.PRECISION_FP64
    raise TypeError(f"expected float32 or float64, got {t.dtype}")


def _check(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def jacobian_raw(field: torch.Tensor, spacing: Sequence[float] = (1.0, 1.0, 1.0),
                 order: int = 4, out: torch.Tensor | None = None) -> torch.Tensor:
    """Jacobian map of one ``[3, nz, ny, nx]`` device field (no autograd),
    into ``out`` (contiguous, ``[nz, ny, nx]``) when given."""
    _check(field, "field")
    if field.dim() != 4 or field.shape[0] != 3:
        raise ValueError("field must have shape (3, nz, ny, nx)")
    _, nz, ny, nx = field.shape
    if out is None:
        J = torch.empty((nz, ny, nx), dtype=field.dtype, device=field.device)
    else:
        _check(out, "out")
        if out.shape != (nz, ny, nx) or out.dtype != field.dtype or out.device != field.device:
            raise ValueError("out must match the field's spatial shape, dtype and device")
        J = out
    with torch.cuda.device(field.device):
        N.check(N.lib.dtb_jacobian_device(_precision(field), order, nx, ny, nz,
                                          *map(float, spacing), field.data_ptr(), J.data_ptr(),
                                          _stream(field)))
    return J


def jacobian_adjoint_raw(field: torch.Tensor, grad_J: torch.Tensor,
                         spacing: Sequence[float] = (1.0, 1.0, 1.0), order: int = 4,
                         out: torch.Tensor | None = None) -> torch.Tensor:
    """(dJ/dfield)^T grad_J for one device field, into ``out`` (contiguous,
    the field's shape) when given."""
    _check(field, "field")
    grad_J = grad_J.contiguous()
    _check(grad_J, "grad_J")
    if grad_J.dtype != field.dtype or grad_J.shape != field.shape[1:]:
        raise ValueError("grad_J must match the field's dtype and spatial shape")
    _, nz, ny, nx = field.shape
    if out is None:
        out = torch.empty_like(field)
    else:
        _check(out, "out")
        if out.shape != field.shape or out.dtype != field.dtype or out.device != field.device:
            raise ValueError("out must match the field's shape, dtype and device")
    with torch.cuda.device(field.device):
        N.check(N.lib.dtb_jacobian_adjoint_device(_precision(field), order, nx, ny, nz,
                                                  *map(float, spacing), field.data_ptr(),
                                                  grad_J.data_ptr(), out.data_ptr(),
                                                  _stream(field)))
    return out


def cof_supported(field: torch.Tensor, order: int = 4) -> bool:
    """Whether the cofactor path takes this field: fourth order, float32,
    rows a multiple of 16 bytes long and a 16-byte-aligned base."""
    return (order == 4 and field.dtype == torch.float32 and field.is_cuda and field.is_contiguous()
            and field.shape[-1] % 4 == 0 and field.data_ptr() % 16 == 0)


def jacobian_cof_raw(field: torch.Tensor, spacing: Sequence[float] = (1.0, 1.0, 1.0),
                     out: torch.Tensor | None = None, cof: torch.Tensor | None = None):
    """Jacobian map of one ``[3, nz, ny, nx]`` device field and the factors
    C[c][a] = cof_ca(I + grad u) * ih_a (``[9, nz, ny, nx]``) its adjoint
    needs: returns ``(J, C)``.  Fourth order; see :func:`cof_supported`."""
    _check(field, "field")
    if field.dim() != 4 or field.shape[0] != 3:
        raise ValueError("field must have shape (3, nz, ny, nx)")
    _, nz, ny, nx = field.shape
    J = torch.empty((nz, ny, nx), dtype=field.dtype, device=field.device) if out is None else out
    Cf = torch.empty((9, nz, ny, nx), dtype=field.dtype, device=field.device) if cof is None else cof
    for t, name in ((J, "out"), (Cf, "cof")):
        _check(t, name)
        if t.dtype != field.dtype or t.device != field.device:
            raise ValueError(f"{name} must match the field's dtype and device")
    if J.shape != (nz, ny, nx) or Cf.shape != (9, nz, ny, nx):
        raise ValueError("out must be (nz, ny, nx) and cof (9, nz, ny, nx)")
    with torch.cuda.device(field.device):
        N.check(N.lib.dtb_jacobian_cof_device(_precision(field), nx, ny, nz, *map(float, spacing),
                                              field.data_ptr(), J.data_ptr(), Cf.data_ptr(), _stream(field)))
    return J, Cf


def jacobian_adjoint_cof_raw(cof: torch.Tensor, grad_J: torch.Tensor,
                             spacing: Sequence[float] = (1.0, 1.0, 1.0),
                             out: torch.Tensor | None = None) -> torch.Tensor:
    """(dJ/dfield)^T grad_J from the factors ``cof`` of
    :func:`jacobian_cof_raw` (no field read), into ``out`` (``[3, nz, ny,
    nx]``) when given."""
    _check(cof, "cof")
    if cof.dim() != 4 or cof.shape[0] != 9:
        raise ValueError("cof must have shape (9, nz, ny, nx)")
    grad_J = grad_J.contiguous()
    if grad_J.data_ptr() % 16:
        grad_J = grad_J.clone()
    _check(grad_J, "grad_J")
    if grad_J.dtype != cof.dtype or grad_J.shape != cof.shape[1:]:
        raise ValueError("grad_J must match cof's dtype and spatial shape")
    _, nz, ny, nx = cof.shape
    if out is None:
        out = torch.empty((3, nz, ny, nx), dtype=cof.dtype, device=cof.device)
    else:
        _check(out, "out")
        if out.shape != (3, nz, ny, nx) or out.dtype != cof.dtype or out.device != cof.device:
            raise ValueError("out must be (3, nz, ny, nx) with cof's dtype and device")
    with torch.cuda.device(cof.device):
        N.check(N.lib.dtb_jacobian_adjoint_cof_device(_precision(cof), nx, ny, nz, *map(float, spacing),
                                                      cof.data_ptr(), grad_J.data_ptr(), out.data_ptr(),
                                                      _stream(cof)))
    return out


def uses_cofactor_path(field: torch.Tensor, order: int = 4) -> bool:
    """Whether :func:`jacobian`'s forward keeps C for its backward: the
    layout allows it (:func:`cof_supported`) and DISPTOOLS_B200_AUTOGRAD is
    not ``weights`` (which asks for the weight pass + gather)."""
    import os
    return os.environ.get("DISPTOOLS_B200_AUTOGRAD", "cofactors") != "weights" and cof_supported(field, order)


class JacobianFunction(torch.autograd.Function):
    """J = det(I + grad u) with the reference stencil (src/jacobian.c:70-242);
    the backward pass is the hand-written adjoint stencil kernel.  For
    float32 fields of a TMA-friendly layout the forward also keeps C =
    cof(I + grad u) * ih (36 bytes a voxel), and the backward is then one
    gather of grad_J * C; otherwise the backward re-reads the field (weight
    pass + gather)."""

    @staticmethod
    def forward(ctx, field, spacing, order):
        ctx.spacing = tuple(float(s) for s in spacing)
        ctx.order = order
        use_cof = ctx.needs_input_grad[0] and uses_cofactor_path(field, order)
        ctx.use_cof = use_cof
        batched = field.dim() == 5
        fields = list(field) if batched else [field]
        J = torch.empty(((field.shape[0],) if batched else ()) + tuple(field.shape[-3:]), dtype=field.dtype,
                        device=field.device)
        Js = list(J) if batched else [J]
        if use_cof:
            Cs = torch.empty(((field.shape[0],) if batched else ()) + (9,) + tuple(field.shape[-3:]),
                             dtype=field.dtype, device=field.device)
            for f, j, cf in zip(fields, Js, list(Cs) if batched else [Cs]):
                jacobian_cof_raw(f, spacing, out=j, cof=cf)
            ctx.save_for_backward(Cs)
        else:
            for f, j in zip(fields, Js):
                jacobian_raw(f, spacing, order, out=j)
            ctx.save_for_backward(field)
        return J

    @staticmethod
    def backward(ctx, grad_J):
        (saved,) = ctx.saved_tensors
        batched = grad_J.dim() == 4
        if ctx.use_cof:
            g = torch.empty(((saved.shape[0],) if batched else ()) + (3,) + tuple(saved.shape[-3:]),
                            dtype=saved.dtype, device=saved.device)
            for cf, gj, gf in zip(list(saved) if batched else [saved], list(grad_J) if batched else [grad_J],
                                  list(g) if batched else [g]):
                jacobian_adjoint_cof_raw(cf, gj, ctx.spacing, out=gf)
            return g, None, None
        field = saved
        if field.dim() == 5:
            g = torch.empty_like(field)
            for f, gj, gf in zip(field, grad_J, g):
                jacobian_adjoint_raw(f, gj, ctx.spacing, ctx.order, out=gf)
        else:
            g = jacobian_adjoint_raw(field, grad_J, ctx.spacing, ctx.order)
        return g, None, None


def jacobian(field: torch.Tensor, spacing: Sequence[float] = (1.0, 1.0, 1.0),
             order: int = 4) -> torch.Tensor:
    """Differentiable Jacobian determinant of ``[3, nz, ny, nx]`` or
    ``[B, 3, nz, ny, nx]`` device fields."""
    field = field.contiguous()
    return JacobianFunction.apply(field, tuple(spacing), order)


def solve(J: torch.Tensor, mask: torch.Tensor, field: torch.Tensor,
          spacing: Sequence[float] = (1.0, 1.0, 1.0), algorithm: str = "gradient", **params):
    """Solve in place on device tensors (``field`` is the initial guess and
    receives the result).  Returns the statistics dict."""
    return solve_batched([(J, mask, field, spacing)], algorithm, **params)[0]


def solve_batched(volumes, algorithm: str = "gradient", **params):
    """Batched in-place solve of ``(J, mask, field[, spacing])`` device
    tensors; all volumes share one dtype (float32 = mixed, float64 = FP64).
    The matching solver takes float64 tensors and solves the volumes one
    after the other (its mask is not used, as by the reference)."""
    vols = list(volumes)
    arr = (N.Volume * len(vols))()
    prec = None
    device = None
    for i, v in enumerate(vols):
        J, mask, field = v[0], v[1], v[2]
        spacing = v[3] if len(v) > 3 else (1.0, 1.0, 1.0)
        for t, n in ((J, "J"), (mask, "mask"), (field, "field")):
            _check(t, n)
        p = _precision(field)
        if prec is not None and p != prec:
            raise TypeError("all volumes must share one dtype")
        prec = p
        device = field.device
        if J.dtype != field.dtype or mask.dtype not in (torch.bool, torch.uint8):
            raise TypeError("J must match the field's dtype and mask must be bool")
        nz, ny, nx = J.shape
        if mask.shape != J.shape or field.shape != (3, nz, ny, nx):
            raise ValueError("shapes of J, mask and field disagree")
        arr[i] = N.Volume(nx, ny, nz, *map(float, spacing), J.data_ptr(), mask.data_ptr(),
                          field.data_ptr())
    p = make_params(**params)
    stats = (N.SolveStats * len(vols))()
    with torch.cuda.device(device):
        N.check(N.lib.dtb_generate_displacement_batched_device(
            N.algorithm_code(algorithm), prec, len(vols), arr, C.byref(p), stats,
            torch.cuda.current_stream(device).cuda_stream))
    return [s.as_dict() for s in stats]
