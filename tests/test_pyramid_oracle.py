"""The CPU restatement of the pyramid filters (oracle/pyramid.py): basic
properties that pin it independently of the device kernels."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyramid as P


def test_gaussian_weights():
    for sigma in (0.5, 1.0, 2.0, 3.3):
        r, w = P.gaussian_weights(sigma)
        assert r == int(np.ceil(4 * sigma)) and len(w) == 2 * r + 1
        assert abs(sum(w) - 1.0) < 1e-15
        assert w == w[::-1]
        assert np.argmax(w) == r
    assert P.gaussian_weights(0.0) == (0, [1.0])


def test_smooth_keeps_constants_and_mass_of_interior_impulse():
    """The sampled filter (method "sampled")."""
    v = np.full((2, 9, 10, 11), 3.25)
    np.testing.assert_allclose(P.smooth(v, (1.0, 2.0, 0.5), "sampled"), v, rtol=1e-15)
    d = np.zeros((1, 31, 31, 31))
    d[0, 15, 15, 15] = 1.0
    s = P.smooth(d, (1.5, 1.0, 2.0), "sampled")
    assert abs(s.sum() - 1.0) < 1e-14
    # separable: the x profile through the centre is the x kernel times the
    # centre weights of y and z
    rx, wx = P.gaussian_weights(1.5)
    _, wy = P.gaussian_weights(1.0)
    _, wz = P.gaussian_weights(2.0)
    prof = s[0, 15, 15, 15 - rx:15 + rx + 1]
    np.testing.assert_allclose(prof, np.array(wx) * wy[len(wy) // 2] * wz[len(wz) // 2], rtol=1e-13)


def test_resample_identity_and_linear_ramp():
    rng = np.random.default_rng(0)
    v = rng.standard_normal((3, 7, 8, 9))
    np.testing.assert_array_equal(P.resample(v, (7, 8, 9)), v)
    np.testing.assert_array_equal(P.resample(v, (7, 8, 9), nearest=True), v)
    # a linear function is reproduced inside the volume
    z, y, x = np.meshgrid(np.arange(12.0), np.arange(10.0), np.arange(14.0), indexing="ij")
    f = (2.0 * x - 0.5 * y + 3.0 * z)[None]
    g = P.resample(f, (5, 4, 6))
    pz, py, px = [np.arange(m) * n / m for n, m in ((12, 5), (10, 4), (14, 6))]
    exact = 2.0 * px[None, None, :] - 0.5 * py[None, :, None] + 3.0 * pz[:, None, None]
    np.testing.assert_allclose(g[0], exact, atol=1e-12)


def test_resample_half_voxel_border():
    """Upsampling 4 -> 8 samples the last output voxel at index 3.5, which
    lies on the image border (n - 0.5) and is outside: it gets 0."""
    v = np.ones((1, 4, 4, 4))
    u = P.resample(v, (8, 8, 8))
    assert np.all(u[0, :7, :7, :7] == 1.0)
    assert np.all(u[0, 7] == 0.0) and np.all(u[0, :, 7] == 0.0) and np.all(u[0, :, :, 7] == 0.0)
    n = P.resample(v, (8, 8, 8), nearest=True)
    np.testing.assert_array_equal(n, u)


def test_resample_keeps_dtype():
    v = np.random.default_rng(1).standard_normal((1, 5, 6, 7)).astype(np.float32)
    assert P.resample(v, (3, 3, 3)).dtype == np.float32
    assert P.smooth(v, (1.0, 1.0, 1.0)).dtype == np.float32


@pytest.mark.parametrize("levels", [1, 2])
def test_driver_runs_and_crops(levels):
    from tests.helpers import ball_problem
    Jt, mask = ball_problem(16, 8, 4, 1.1)
    out = P.displacement(Jt, mask=mask, levels=levels, it_max=5)
    assert out.shape == (3, 16, 16, 16)
    assert np.isfinite(out).all()


def test_blob_problem_device_matches_numpy_on_cpu():
    from disptools_b200.synthetic import blob_problem, blob_problem_device
    J, m = blob_problem((23, 19, 27), blobs=5, seed=4, sigma=(2.0, 5.0))
    Jd, md = blob_problem_device((23, 19, 27), blobs=5, seed=4, sigma=(2.0, 5.0), device="cpu")
    np.testing.assert_allclose(Jd.numpy(), J, rtol=1e-14)
    np.testing.assert_array_equal(md.numpy(), m)


def test_level_geometry_follows_the_reference_rule():
    """disptools/displacements.py:459-466: each level halves the previous
    size (integer division); spacings keep the finest level's extent."""
    from disptools_b200.pyramid import level_geometry
    sizes, spacings = level_geometry((386, 514, 514), (1.0, 1.0, 1.0), 3)
    assert sizes == [(386, 514, 514), (193, 257, 257), (96, 128, 128)]
    assert spacings[1] == (2.0, 2.0, 2.0)
    assert spacings[2] == (514 / 128, 514 / 128, 386 / 96)
    sizes, spacings = level_geometry((7, 9, 11), (0.5, 1.5, 2.0), 2)
    assert sizes == [(7, 9, 11), (3, 4, 5)]
    assert spacings[1] == (0.5 * 11 / 5, 1.5 * 9 / 4, 2.0 * 7 / 3)


def test_pyramid_rejects_levels_below_three_voxels_before_device_work():
    import numpy as np
    import pytest
    from disptools_b200 import pyramid
    with pytest.raises(ValueError, match="below 3"):
        pyramid.displacement(np.ones((5, 5, 5)), levels=3)


# --- the recursive Gaussian (Deriche, INRIA RR-1893, 1993) ------------------
# ITK is not installed, so the filter is pinned by its defining properties.

def _impulse_response(sigma, n=None):
    n = n or int(40 * sigma) + 41
    d = np.zeros((1, 1, 1, n))
    d[0, 0, 0, n // 2] = 1.0
    return P.smooth(d, (sigma, 0.0, 0.0))[0, 0, 0], n // 2


@pytest.mark.parametrize("sigma", [0.5, 1.0, 2.0, 4.0, 8.0, 16.0])
def test_recursive_impulse_response_is_a_gaussian(sigma):
    """Deriche's fourth-order fit of the Gaussian: the impulse response
    matches the sampled Gaussian exp(-k^2 / (2 sigma^2)) / sum to within
    1e-3 of its peak, sums to 1 and is symmetric."""
    h, c = _impulse_response(sigma)
    k = np.arange(h.size) - c
    g = np.exp(-k * k / (2.0 * sigma * sigma))
    g /= g.sum()
    assert np.max(np.abs(h - g)) <= 1e-3 * g.max()
    assert abs(h.sum() - 1.0) <= 1e-12
    np.testing.assert_allclose(h, h[::-1], atol=1e-14)


def test_recursive_unit_gain_and_constants():
    for sigma in (0.7, 2.0, 5.5):
        n, m, d, gc, ga = P.deriche_coefficients(sigma)
        den = 1.0 + sum(d)
        assert abs((sum(n) + sum(m)) / den - 1.0) <= 1e-12
        assert abs(gc + ga - 1.0) <= 1e-12
    v = np.full((2, 7, 9, 11), -1.75)
    np.testing.assert_allclose(P.smooth(v, (1.0, 2.0, 3.0)), v, rtol=1e-12)
    np.testing.assert_allclose(P.smooth(v.astype(np.float32), (1.0, 2.0, 3.0)), v, rtol=1e-6)


@pytest.mark.parametrize("sigma", [1.0, 2.5, 6.0])
def test_recursive_zero_flux_border(sigma):
    """Each recursion starts in the steady state of its border value: the
    result equals that of the signal continued with its edge values far
    beyond both ends, cropped."""
    x = np.random.default_rng(int(sigma * 10)).standard_normal(37)
    pad = int(30 * sigma)
    xp = np.concatenate([np.full(pad, x[0]), x, np.full(pad, x[-1])])
    a = P.smooth(x[None, None, None], (sigma, 0.0, 0.0))[0, 0, 0]
    b = P.smooth(xp[None, None, None], (sigma, 0.0, 0.0))[0, 0, 0, pad:-pad]
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-10)


def test_recursive_separable_linear_and_axis_order():
    rng = np.random.default_rng(4)
    u, w = rng.standard_normal((2, 1, 8, 9, 10))
    s = (1.2, 0.8, 2.0)
    np.testing.assert_allclose(P.smooth(2.0 * u - 3.0 * w, s), 2.0 * P.smooth(u, s) - 3.0 * P.smooth(w, s),
                               atol=1e-12)
    # sigma 0 leaves an axis alone; the passes commute up to rounding
    np.testing.assert_array_equal(P.smooth(u, (0.0, 0.0, 0.0)), u)
    ax = P.smooth(P.smooth(u, (0.0, 0.0, s[2])), (s[0], s[1], 0.0))
    np.testing.assert_allclose(P.smooth(u, s), ax, atol=1e-12)


def test_recursive_close_to_sampled_filter():
    v = np.random.default_rng(9).standard_normal((1, 12, 13, 14))
    a = P.smooth(v, (2.0, 1.5, 1.0))
    b = P.smooth(v, (2.0, 1.5, 1.0), "sampled")
    assert np.max(np.abs(a - b)) <= 5e-3 * np.max(np.abs(v))
