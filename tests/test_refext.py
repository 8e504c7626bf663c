"""The reference's own NumPy extension (python_c_extension/_disptools.c),
compiled unchanged with CUDA support and linked against the drop-in library
(oracle/Makefile, target ``refext``): the boundary a user of the reference
would switch to.

CPU tests: the module loads with every name resolved; the names the drop-in
does not replace (the CPU solvers, the shape descriptors) come from the
reference's own objects and reproduce config 1; an error raised inside the
drop-in reaches the extension's error check.  GPU tests: ``displacement``
with ``gpu_id = 0`` runs the drop-in's ``generate_displacement_*_cuda`` and
reproduces config 1; ``jacobian`` and ``regularise`` go through the
drop-in's ``jacobian_dynamic`` and ``regularise``."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from oracle.oracle import Reference, reference_extension
from tests.helpers import ball_problem, masked_max

EXT = reference_extension()
pytestmark = pytest.mark.skipif(EXT is None, reason="reference extension not built (oracle/Makefile refext)")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# reference defaults, src/headers/disptools.h and disptools/displacements.py:238-260
ARGS = [9.99e-4, 0.2, 0.1, 0.4, 1.2, 0.5, 0.1, 1e-3, 10.0, 1e-6, 1e-9, False, 1000]


def _dropin():
    """The drop-in library instance the extension is linked to (the same
    mapping: dlopen of one path returns one handle)."""
    lib = C.CDLL(os.path.join(ROOT, "disptools_b200", "libdisptools_b200.so"))
    lib.dtb_set_default_precision.argtypes = [C.c_int]
    lib.dtb_set_default_precision.restype = C.c_int
    return lib


def _linked_libraries():
    maps = open("/proc/self/maps").read()
    return {ln.split()[-1] for ln in maps.splitlines() if ln.endswith(".so") or ".so." in ln}


def test_reference_extension_links_the_dropin():
    libs = _linked_libraries()
    assert any(p.endswith("disptools_b200/libdisptools_b200.so") for p in libs), libs
    assert EXT.get_float_type_size() == 64


def test_cpu_solver_through_reference_objects(golden):
    """gpu_id < 0: the reference's own CPU solver, linked beside the drop-in."""
    Jt, mask = ball_problem(40, 20, 10)
    c1 = golden["cases"]["config1"]
    f = np.zeros((3, 40, 40, 40))
    assert EXT.displacement((1.0, 1.0, 1.0), Jt, mask, *ARGS, f, "gradient", -1) is None
    ref = Reference("ref64")
    assert masked_max(ref.jacobian(f), Jt, mask) == pytest.approx(c1["masked_max"], rel=1e-9)
    np.testing.assert_allclose(f[:, 20, 20, :], np.array(c1["field_line"]), atol=1e-12)


def test_shape_descriptor_from_reference_objects():
    # a cube scores higher on cubeness, an octahedron on octahedroness
    # (src/shape_descriptors.c:25-150; boolean images)
    z, y, x = np.meshgrid(*[np.arange(20)] * 3, indexing="ij")
    cube = (abs(x - 10) < 5) & (abs(y - 10) < 5) & (abs(z - 10) < 5)
    octa = abs(x - 10) + abs(y - 10) + abs(z - 10) < 7
    c = [EXT.shape_descriptor(im, (10.0, 10.0, 10.0), (1.0, 1.0, 1.0), "cubeness") for im in (cube, octa)]
    o = [EXT.shape_descriptor(im, (10.0, 10.0, 10.0), (1.0, 1.0, 1.0), "octahedroness") for im in (cube, octa)]
    assert c[0] > o[0] and o[1] > c[1]
    assert 0.9 < c[0] < 1.1 and 0.9 < o[1] < 1.1


@pytest.mark.gpu
def test_gpu_solver_through_dropin(golden, oracle):
    """gpu_id = 0: generate_displacement_gradient_cuda of the drop-in, FP64
    device path, against the reference's config-1 result; then the default
    mixed path within 1e-4 of its residual."""
    lib = _dropin()
    Jt, mask = ball_problem(40, 20, 10)
    c1 = golden["cases"]["config1"]
    prev = lib.dtb_set_default_precision(1)  # DTB_PRECISION_FP64
    try:
        f = np.zeros((3, 40, 40, 40))
        EXT.displacement((1.0, 1.0, 1.0), Jt, mask, *ARGS, f, "gradient", 0)
        fg = np.zeros((3, 40, 40, 40))
        EXT.displacement((1.0, 1.0, 1.0), Jt, mask, *ARGS[:-1], 30, fg, "greedy", 0)
    finally:
        lib.dtb_set_default_precision(prev)
    assert masked_max(oracle.jacobian(f), Jt, mask) == pytest.approx(c1["masked_max"], rel=1e-9)
    np.testing.assert_allclose(f[:, 20, 20, :], np.array(c1["field_line"]), atol=1e-12)
    refg, _ = oracle.solve("greedy", Jt, mask, it_max=30)
    assert np.max(np.abs(fg - refg)) <= 1e-10
    f32 = np.zeros((3, 40, 40, 40))
    EXT.displacement((1.0, 1.0, 1.0), Jt, mask, *ARGS, f32, "gradient", 0)
    assert abs(masked_max(oracle.jacobian(f32), Jt, mask) - c1["masked_max"]) <= 1e-4


@pytest.mark.gpu
def test_gpu_jacobian_and_regularise_through_dropin(golden):
    g = golden["jacobian"]
    for k in ("sin10", "rand0", "rand1"):
        f = np.ascontiguousarray(g[f"{k}_field"])
        sp = tuple(g[f"{k}_spacing"]) if f"{k}_spacing" in g else (1.0, 1.0, 1.0)
        out = np.zeros(f.shape[1:])
        EXT.jacobian(sp, f, out)
        ref = g[f"{k}_J"]
        assert np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-12, k
    ref = g["rand0_J"]
    J = ref.copy()
    J.flat[::7] = -0.5
    want = Reference("ref64").regularise(J, 0.1)
    got = J.copy()
    EXT.regularise(got, 0.1)
    np.testing.assert_array_equal(got, want)


def test_dropin_error_reaches_extension():
    """An argument error inside the drop-in (a 2-voxel axis) is reported
    through the drop-in's error state, which the extension checks."""
    Jt = np.ones((2, 5, 5))
    mask = np.ones((2, 5, 5), dtype=np.bool_)
    f = np.zeros((3, 2, 5, 5))
    with pytest.raises((RuntimeError, ValueError)):
        EXT.displacement((1.0, 1.0, 1.0), Jt, mask, *ARGS, f, "gradient", 0)
