"""NumPy-level API over the C ABI.

Arrays use the reference library layout (src/headers/disptools.h:30-36 of
disptools): fields ``[3, nz, ny, nx]``, scalar maps ``[nz, ny, nx]``, masks
``bool``.  Host arrays are float64 (FLOATING = double at the ABI); the
device precision is chosen per call (``"mixed"``: FP32 field and stencils
with FP64 reductions; ``"fp64"``: FP64 throughout).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

import numpy as np

from . import _native as N

# Defaults of the reference Python wrapper (disptools/displacements.py:238-260).
DEFAULTS = dict(epsilon=9.99e-4, tolerance=0.2, eta=0.1, eta_max=0.4, alpha=1.2, beta=0.5,
                gamma=0.1, delta=1e-3, zeta=10.0, theta=1e-6, iota=1e-9, strict=False,
                it_max=50000)


def make_params(**kw) -> N.Params:
    unknown = set(kw) - set(DEFAULTS)
    if unknown:
        raise TypeError(f"unknown solver parameters: {sorted(unknown)}")
    p = {**DEFAULTS, **kw}
    out = N.Params()
    for k in ("epsilon", "tolerance", "eta", "eta_max", "alpha", "beta", "gamma", "delta",
              "zeta", "theta", "iota"):
        setattr(out, k, float(p[k]))
    out.strict = 1 if p["strict"] else 0
    out.it_max = int(p["it_max"])
    return out


def _f64(a, name, shape=None) -> np.ndarray:
    a = np.asarray(a)
    if a.dtype != np.float64:
        raise TypeError(f"{name} must be float64 (got {a.dtype})")
    if not a.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)} (got {a.shape})")
    return a


def _mask(m, shape) -> np.ndarray:
    m = np.asarray(m)
    if m.dtype != np.bool_:
        raise TypeError(f"mask must be bool (got {m.dtype})")
    if not m.flags.c_contiguous or m.shape != tuple(shape):
        raise ValueError(f"mask must be C-contiguous with shape {tuple(shape)}")
    return m


def jacobian(field: np.ndarray, spacing: Sequence[float] = (1.0, 1.0, 1.0)) -> np.ndarray:
    """Jacobian determinant map of a ``[3, nz, ny, nx]`` float64 field
    (``jacobian_dynamic``, src/jacobian.c:7-21), computed on the GPU in FP64."""
    field = _f64(field, "field")
    if field.ndim != 4 or field.shape[0] != 3:
        raise ValueError("field must have shape (3, nz, ny, nx)")
    _, nz, ny, nx = field.shape
    J = np.empty((nz, ny, nx), np.float64)
    N.lib.jacobian_dynamic(nx, ny, nz, *map(float, spacing), field.ctypes.data, J.ctypes.data)
    if N.lib.disptools_has_error():
        N.check(N.ERR_CUDA)
    return J


def regularise(J: np.ndarray, epsilon: float) -> np.ndarray:
    """Copy of ``J`` with values below ``epsilon`` replaced by ``epsilon``
    (src/jacobian.c:29-55)."""
    J = _f64(J, "J").copy()
    nz, ny, nx = J.shape
    N.lib.regularise(nx, ny, nz, J.ctypes.data, float(epsilon))
    if N.lib.disptools_has_error():
        N.check(N.ERR_CUDA)
    return J


def solve(J: np.ndarray, mask: np.ndarray, field: np.ndarray | None = None,
          spacing: Sequence[float] = (1.0, 1.0, 1.0), algorithm: str = "gradient",
          precision: str = "mixed", **params):
    """Generate a displacement field whose Jacobian matches ``J`` in ``mask``.

    Returns ``(field, stats)``.  ``field`` (optional) is the initial guess; it
    is not modified."""
    J = _f64(J, "J")
    if J.ndim != 3:
        raise ValueError("J must have shape (nz, ny, nx)")
    nz, ny, nx = J.shape
    mask = _mask(mask, J.shape)
    out = (np.zeros((3, nz, ny, nx)) if field is None
           else _f64(field, "field", (3, nz, ny, nx)).copy())
    p = make_params(**params)
    st = N.SolveStats()
    rc = N.lib.dtb_generate_displacement(N.algorithm_code(algorithm), N.precision_code(precision),
                                         nx, ny, nz, *map(float, spacing), J.ctypes.data,
                                         mask.ctypes.data, C.byref(p), out.ctypes.data,
                                         C.byref(st))
    N.check(rc)
    return out, st.as_dict()


def solve_batched(volumes: Iterable, algorithm: str = "gradient", precision: str = "mixed",
                  inplace: bool = False, **params):
    """Solve several independent volumes of any sizes in one batched run.

    ``volumes`` is an iterable of ``(J, mask)``, ``(J, mask, field)`` or
    ``(J, mask, field, spacing)`` tuples.  Returns a list of
    ``(field, stats)``.  With ``inplace`` each given field (C-contiguous
    float64) is the initial guess and receives the result, as the reference
    C API's in/out field does, with no copy; fields in pinned memory then
    move at full link speed."""
    vols = list(volumes)
    arr = (N.Volume * len(vols))()
    keep = []
    outs = []
    for i, v in enumerate(vols):
        J, mask = v[0], v[1]
        field = v[2] if len(v) > 2 else None
        spacing = v[3] if len(v) > 3 else (1.0, 1.0, 1.0)
        J = _f64(J, "J")
        nz, ny, nx = J.shape
        mask = _mask(mask, J.shape)
        if inplace:
            if (not isinstance(field, np.ndarray) or field.dtype != np.float64
                    or not field.flags.c_contiguous or field.shape != (3, nz, ny, nx)):
                raise ValueError("inplace needs C-contiguous float64 fields of shape (3, nz, ny, nx)")
            out = field
        else:
            out = (np.zeros((3, nz, ny, nx)) if field is None
                   else _f64(field, "field", (3, nz, ny, nx)).copy())
        keep += [J, mask]
        outs.append(out)
        arr[i] = N.Volume(nx, ny, nz, *map(float, spacing), J.ctypes.data, mask.ctypes.data,
                          out.ctypes.data)
    p = make_params(**params)
    stats = (N.SolveStats * len(vols))()
    rc = N.lib.dtb_generate_displacement_batched(N.algorithm_code(algorithm),
                                                 N.precision_code(precision), len(vols), arr,
                                                 C.byref(p), stats)
    N.check(rc)
    return [(o, s.as_dict()) for o, s in zip(outs, stats)]


def set_verbose(on: bool) -> bool:
    """Print the reference's per-iteration lines on stdout after each solve;
    returns the previous setting."""
    return bool(N.lib.dtb_set_verbose(1 if on else 0))


def set_autotune(on: bool) -> bool:
    """Turn the tile-shape autotuner of gradient solves on or off; returns
    the previous setting."""
    return bool(N.lib.dtb_set_autotune(1 if on else 0))


TRIAL_KERNELS = ("formed", "release")


def tile_config() -> dict:
    """Tile shape of the last solve on the current device, and its trial
    kernel: "formed" (candidate planes formed in a shared ring, one block
    barrier per plane) or "release" (no barrier in the plane loop)."""
    a = (C.c_int * 4)()
    N.check(N.lib.dtb_get_tile_config(a))
    kind = N.lib.dtb_get_trial_kernel()
    N.check(min(kind, 0))
    return {"tile_x": a[0], "trial_threads_y": a[1], "gradient_threads_y": a[2], "bz": a[3],
            "trial_kernel": TRIAL_KERNELS[kind]}


def release_device_memory() -> None:
    """Free the device memory the library keeps between calls on the current
    device (workspace and staging area); the next call allocates again."""
    N.check(N.lib.dtb_release_device_memory())


def set_default_precision(precision) -> None:
    """Device precision used by the reference-named entry points."""
    N.check(N.lib.dtb_set_default_precision(N.precision_code(precision)))


def kernel_launch_count() -> int:
    return int(N.lib.dtb_kernel_launch_count())


def set_profiling(on: bool) -> None:
    """Start (clearing the counters) or stop per-kernel profiling."""
    N.lib.dtb_set_profiling(1 if on else 0)


def kernel_profile() -> dict:
    """{kernel: (launches that did work, total device ms)} since profiling
    was switched on."""
    arr = (N.KernelProfile * 8)()
    n = N.lib.dtb_get_profile(arr, 8)
    return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(n)}
