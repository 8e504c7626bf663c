"""Field files (RVF, legacy VTK): round trips, the header formats, error
cases, and files exchanged with the reference's own readers and writers
(src/rvf_io.c, src/vtk_io.c compiled into oracle/_ref) when that build is
present."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from disptools_b200 import io as fio

REF_IO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "libdisptools_ref64_io.so")


def _field(shape, nd=3, seed=0):
    f = np.random.default_rng(seed).standard_normal((nd,) + shape)
    f.flat[0] = 0.0  # leading zero bytes (see test_reference_reads_our_rvf)
    return f


def test_rvf_round_trip_and_header(tmp_path):
    f = _field((5, 6, 7))
    p = tmp_path / "a.rvf"
    fio.write_rvf(p, f, (0.5, 1.25, 2.0))
    with open(p, "rb") as fh:
        assert fh.readline() == b"7 6 5\n"
        assert fh.readline() == b"0.500000 1.250000 2.000000\n"
        raw = np.frombuffer(fh.read(), dtype=np.float64)
    np.testing.assert_array_equal(raw, f.reshape(3, -1).T.ravel())
    g, sp = fio.read_rvf(p)
    np.testing.assert_array_equal(g, f)
    assert sp == (0.5, 1.25, 2.0)


def test_rvf_spacing_goes_through_float(tmp_path):
    p = tmp_path / "s.rvf"
    fio.write_rvf(p, _field((3, 3, 3)), (0.1, 1.0 / 3.0, 7.0))
    _, sp = fio.read_rvf(p)
    assert sp == tuple(float(np.float32(v)) for v in (0.1, 0.333333, 7.0))


@pytest.mark.parametrize("nd", [1, 3])
def test_vtk_round_trip_and_header(tmp_path, nd):
    f = _field((4, 3, 5), nd=nd, seed=nd)
    p = tmp_path / "a.vtk"
    fio.write_vtk(p, f, (1.0, 2.0, 0.25))
    with open(p, "rb") as fh:
        head = [fh.readline() for _ in range(10)]
        raw = np.frombuffer(fh.read(), dtype=">f8")
    assert head[0] == b"# vtk DataFile Version 3.0\n" and head[2] == b"BINARY\n"
    assert head[4] == b"DIMENSIONS 5 3 4\n" and head[6] == b"SPACING 1.000000 2.000000 0.250000\n"
    assert head[7] == b"POINT_DATA 60\n" and head[8] == f"SCALARS image_data double {nd}\n".encode()
    assert head[9].startswith(b"L")
    np.testing.assert_array_equal(raw, f.reshape(nd, -1).T.ravel())
    g, sp = fio.read_vtk(p)
    np.testing.assert_array_equal(g, f)
    assert sp == (1.0, 2.0, 0.25)


def test_io_errors(tmp_path):
    with pytest.raises(OSError):
        fio.read_rvf(tmp_path / "missing.rvf")
    p = tmp_path / "short.rvf"
    fio.write_rvf(p, _field((3, 4, 5)))
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])
    with pytest.raises(OSError):
        fio.read_rvf(p)
    q = tmp_path / "f.vtk"
    fio.write_vtk(q, _field((3, 3, 3), nd=1))
    txt = open(q, "rb").read().replace(b"image_data double", b"image_data float")
    open(q, "wb").write(txt)
    with pytest.raises(OSError):
        fio.read_vtk(q)
    with pytest.raises(ValueError):
        fio.write_rvf(tmp_path / "x.rvf", np.zeros((2, 3, 3, 3)))


class _Image(C.Structure):
    """The reference's Image (src/headers/disptools.h:294-303), FLOATING = double."""
    _fields_ = [("nd", C.c_size_t), ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("data", C.POINTER(C.c_double))]


@pytest.fixture(scope="module")
def ref_io():
    if not os.path.exists(REF_IO):
        pytest.skip("reference file readers not built (oracle/Makefile ref)")
    lib = C.CDLL(REF_IO)
    for name in ("write_rvf", "write_vtk"):
        getattr(lib, name).argtypes = [C.c_char_p, _Image]
        getattr(lib, name).restype = C.c_int
    for name in ("read_rvf", "read_vtk"):
        getattr(lib, name).argtypes = [C.c_char_p, C.POINTER(_Image)]
        getattr(lib, name).restype = C.c_int
    lib.delete_image.argtypes = [C.POINTER(_Image)]
    return lib


def _to_image(a, spacing):
    a = np.ascontiguousarray(a, dtype=np.float64)
    nd, nz, ny, nx = a.shape
    return _Image(nd, nx, ny, nz, *spacing, a.ctypes.data_as(C.POINTER(C.c_double))), a


def _from_image(lib, img):
    n = img.nd * img.nz * img.ny * img.nx
    a = np.ctypeslib.as_array(img.data, shape=(n,)).copy().reshape(img.nd, img.nz, img.ny, img.nx)
    sp = (img.dx, img.dy, img.dz)
    lib.delete_image(C.byref(img))
    return a, sp


@pytest.mark.parametrize("fmt", ["rvf", "vtk"])
def test_reference_reads_our_files(tmp_path, ref_io, fmt):
    """Our writers, the reference's readers.  The reference's RVF reader
    skips whitespace bytes at the start of the binary data (its header
    fscanf ends in "\\n"), so the field starts with a zero."""
    f = _field((4, 5, 6), seed=3)
    p = tmp_path / f"a.{fmt}"
    (fio.write_rvf if fmt == "rvf" else fio.write_vtk)(p, f, (0.75, 1.0, 1.5))
    img = _Image()
    assert getattr(ref_io, f"read_{fmt}")(os.fsencode(p), C.byref(img)) == 0
    a, sp = _from_image(ref_io, img)
    np.testing.assert_array_equal(a, f)
    assert sp == (0.75, 1.0, 1.5)


@pytest.mark.parametrize("fmt", ["rvf", "vtk"])
def test_we_read_reference_files(tmp_path, ref_io, fmt):
    f = _field((3, 7, 5), seed=4)
    p = tmp_path / f"b.{fmt}"
    img, keep = _to_image(f, (2.0, 0.5, 1.0))
    assert getattr(ref_io, f"write_{fmt}")(os.fsencode(p), img) == 0
    g, sp = (fio.read_rvf if fmt == "rvf" else fio.read_vtk)(p)
    np.testing.assert_array_equal(g, f)
    assert sp == (2.0, 0.5, 1.0)
