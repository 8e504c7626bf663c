"""Field files: RVF and legacy VTK, through the library's C ABI.

The formats are those of the reference C library (src/rvf_io.c,
src/vtk_io.c); arrays are in this package's layout, ``[C, nz, ny, nx]``
float64, with the spacing as (dx, dy, dz).  ``read_rvf`` replaces the
reference's Python reader (disptools/io.py:167-191), which returns a
SimpleITK image.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence, Tuple

import numpy as np

from . import _native as N


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def write_rvf(filename, field: np.ndarray, spacing: Sequence[float] = (1.0, 1.0, 1.0)) -> None:
    """Write a ``[3, nz, ny, nx]`` field to an RVF file."""
    f = np.ascontiguousarray(field, dtype=np.float64)
    if f.ndim != 4 or f.shape[0] != 3:
        raise ValueError("field must be [3, nz, ny, nx]")
    _, nz, ny, nx = f.shape
    N.check(N.lib.dtb_write_rvf(_path(filename), nx, ny, nz, *map(float, spacing), f.ctypes.data))


def read_rvf(filename) -> Tuple[np.ndarray, Tuple[float, float, float]]:
    """Read an RVF file: (field ``[3, nz, ny, nx]``, spacing (dx, dy, dz))."""
    n = [C.c_size_t() for _ in range(3)]
    d = [C.c_double() for _ in range(3)]
    N.check(N.lib.dtb_read_rvf_header(_path(filename), *map(C.byref, n), *map(C.byref, d)))
    nx, ny, nz = (v.value for v in n)
    out = np.empty((3, nz, ny, nx))
    N.check(N.lib.dtb_read_rvf(_path(filename), out.ctypes.data, out.size))
    return out, tuple(v.value for v in d)


def write_vtk(filename, data: np.ndarray, spacing: Sequence[float] = (1.0, 1.0, 1.0)) -> None:
    """Write a ``[C, nz, ny, nx]`` (or ``[nz, ny, nx]``) array to a legacy
    VTK file (STRUCTURED_POINTS, big-endian doubles)."""
    a = np.ascontiguousarray(data, dtype=np.float64)
    if a.ndim == 3:
        a = a[None]
    if a.ndim != 4:
        raise ValueError("data must be [C, nz, ny, nx] or [nz, ny, nx]")
    c, nz, ny, nx = a.shape
    N.check(N.lib.dtb_write_vtk(_path(filename), c, nx, ny, nz, *map(float, spacing), a.ctypes.data))


def read_vtk(filename) -> Tuple[np.ndarray, Tuple[float, float, float]]:
    """Read a legacy VTK file written as above: (data ``[C, nz, ny, nx]``,
    spacing (dx, dy, dz))."""
    nd = C.c_int()
    n = [C.c_size_t() for _ in range(3)]
    d = [C.c_double() for _ in range(3)]
    N.check(N.lib.dtb_read_vtk_header(_path(filename), C.byref(nd), *map(C.byref, n),
                                      *map(C.byref, d)))
    nx, ny, nz = (v.value for v in n)
    out = np.empty((nd.value, nz, ny, nx))
    N.check(N.lib.dtb_read_vtk(_path(filename), out.ctypes.data, out.size))
    return out, tuple(v.value for v in d)
