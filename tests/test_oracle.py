"""The CPU oracle against the reference's golden vectors and the reference
library itself (CPU only)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Reference
from tests.helpers import ball_problem, masked_max

pytestmark = pytest.mark.filterwarnings("ignore::DeprecationWarning")


def test_jacobian_matches_golden(oracle, oracle_pd2, golden):
    g = golden["jacobian"]
    np.testing.assert_array_equal(oracle.jacobian(g["sin10_field"]), g["sin10_J"])
    np.testing.assert_array_equal(oracle.jacobian(g["i2_field"], (2.0, 3.0, 4.0)), g["i2_J"])
    for k in range(4):
        f, sp = g[f"rand{k}_field"], tuple(g[f"rand{k}_spacing"])
        np.testing.assert_array_equal(oracle.jacobian(f, sp), g[f"rand{k}_J"])
        np.testing.assert_array_equal(oracle_pd2.jacobian(f, sp), g[f"rand{k}_J_pd2"])


def test_one_sided_macros_known_answers(oracle):
    """test/c/test_jacobian_macros.cpp:70-148: forward second-order
    differences of i*i data on a 5x6x7 grid at voxel (2, 1, 3)."""
    lib = oracle.lib
    lib.oracle_fd.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, C.c_double]
    lib.oracle_fd.restype = C.c_double
    nx, ny, nz = 5, 6, 7
    spacing = (2.0, 3.0, 4.0)
    i = np.arange(3 * nz * ny * nx, dtype=np.float64)
    data = i * i
    p = (2, 1, 3)
    strides = (1, nx, nx * ny)
    for comp in range(3):
        base = data[comp * nz * ny * nx:]
        o = p[2] * nx * ny + p[1] * nx + p[0]
        for axis in range(3):
            s = strides[axis]
            want = (1.0 / spacing[comp]) * (-1.5 * base[o] + 2.0 * base[o + s] - 0.5 * base[o + 2 * s])
            got = lib.oracle_fd(base.ctypes.data, o, s, 0, 1.0 / spacing[comp])
            assert abs(got - want) <= 1e-6


def test_jacobian_of_smooth_field_analytic(oracle, golden):
    """Stands in for test/test_displacements.py:43-55 (which compares with
    ITK): the field u_c = sin(r^2) on linspace(0, 0.5, 10) has
    det(I + grad u) = 1 + sum_a du/dx_a, checked on the interior at rtol 1e-3."""
    n = 10
    f = golden["jacobian"]["sin10_field"]
    J = oracle.jacobian(f)
    x = np.linspace(0, 0.5, n)
    h = x[1] - x[0]
    xx, yy, zz = np.meshgrid(x, x, x)
    c = np.cos(xx ** 2 + yy ** 2 + zz ** 2)
    exact = 1.0 + 2.0 * c * (xx + yy + zz) * h
    inner = (slice(1, n - 1),) * 3
    assert np.allclose(J[inner], exact[inner], rtol=1e-3)


def test_solver_matches_golden(oracle, golden):
    sol = golden["solver"]
    for case in golden["cases"]["cases"]:
        k = case["name"]
        out, st = oracle.solve(case["algorithm"], sol[f"{k}_Jt"], sol[f"{k}_mask"],
                               field=sol[f"{k}_field0"], spacing=tuple(case["spacing"]),
                               **case["params"])
        np.testing.assert_array_equal(out, sol[f"{k}_out"], err_msg=k)


def test_config1_matches_golden(oracle, golden):
    Jt, mask = ball_problem(40, 20, 10)
    out, st = oracle.solve("gradient", Jt, mask, it_max=1000)
    c1 = golden["cases"]["config1"]
    assert st.iterations == 123 and st.reason == "tolerance reached"
    assert masked_max(oracle.jacobian(out), Jt, mask) == pytest.approx(c1["masked_max"], rel=1e-12)
    assert st.max_error == pytest.approx(c1["masked_max"], rel=1e-12)
    np.testing.assert_allclose(out[:, 20, 20, :], np.array(c1["field_line"]), rtol=0, atol=1e-14)


def test_compute_error_semantics(oracle):
    """src/headers/error.h:128-150: full error in the mask, tolerance band
    outside it, max only over the mask."""
    Jt = np.array([1.0, 1.0, 1.0, 1.0]).reshape(1, 1, 4)
    Jf = np.array([1.3, 1.3, 0.7, 1.05]).reshape(1, 1, 4)
    mask = np.array([True, False, False, False]).reshape(1, 1, 4)
    tot, mx, v = oracle.compute_error(Jt, Jf, mask, 0.2)
    np.testing.assert_allclose(v.ravel(), [0.3, 0.1, -0.1, 0.0], atol=1e-15)
    assert mx == pytest.approx(0.3)
    assert tot == pytest.approx(0.09 + 0.01 + 0.01)


def test_planted_mistake_is_detected(oracle_pd2, golden):
    """The comparison is sensitive: the second-order oracle does not pass the
    fourth-order golden vectors."""
    g = golden["jacobian"]
    f, sp = g["rand2_field"], tuple(g["rand2_spacing"])
    assert not np.array_equal(oracle_pd2.jacobian(f, sp), g["rand2_J"])


@pytest.mark.skipif(not Reference.available("ref64"), reason="reference build not present")
def test_oracle_matches_live_reference(oracle):
    ref = Reference("ref64")
    rng = np.random.default_rng(7)
    for shape in [(3, 3, 3), (3, 4, 5), (6, 5, 4), (16, 9, 21)]:
        f = rng.normal(scale=0.2, size=(3,) + shape)
        sp = tuple(rng.uniform(0.5, 2.0, 3))
        np.testing.assert_array_equal(oracle.jacobian(f, sp), ref.jacobian(f, sp))
    Jt, mask = ball_problem(16, 8, 4, 0.9)
    f0 = rng.normal(scale=0.02, size=(3, 16, 16, 16))
    for alg in ("gradient", "greedy"):
        a, _ = oracle.solve(alg, Jt, mask, field=f0, it_max=60, strict=(alg == "gradient"))
        b = ref.solve(alg, Jt, mask, field=f0, it_max=60, strict=(alg == "gradient"))
        np.testing.assert_array_equal(a, b)
