"""Multi-resolution pyramid on the device against its CPU restatement
(oracle/pyramid.py): the smoothing and resampling kernels bit for bit, the
driver through the FP64 solver to 1e-10, the mixed path by the residual
rule, the matching solver against the reference's own at every level."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from disptools_b200 import pyramid as D
from oracle import pyramid as P
from tests.helpers import ball_problem, masked_max

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("comps,shape,sigma", [
    (1, (13, 17, 11), (1.0, 1.0, 1.0)),
    (3, (9, 10, 23), (2.0, 0.7, 1.3)),
    (1, (5, 6, 4), (0.0, 3.0, 0.5)),
])
@pytest.mark.parametrize("method", ["recursive", "sampled"])
def test_smooth_bitwise(dtype, comps, shape, sigma, method):
    v = np.random.default_rng(comps).standard_normal((comps,) + shape).astype(dtype)
    got = D.smooth(torch.from_numpy(v).cuda(), sigma, method).cpu().numpy()
    np.testing.assert_array_equal(got, P.smooth(v, sigma, method))


def test_recursive_smooth_long_lines_bitwise():
    """Lines longer than the filter's memory along every axis, large sigma
    (the config-5 level sizes' scale), FP32."""
    v = np.random.default_rng(8).standard_normal((1, 40, 70, 130)).astype(np.float32)
    sig = (8.0, 4.0, 2.0)
    got = D.smooth(torch.from_numpy(v).cuda(), sig).cpu().numpy()
    np.testing.assert_array_equal(got, P.smooth(v, sig))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("nearest", [False, True])
@pytest.mark.parametrize("src,dst", [
    ((13, 17, 11), (6, 8, 5)),
    ((6, 8, 5), (13, 17, 11)),
    ((8, 8, 8), (16, 16, 16)),
    ((10, 9, 12), (10, 9, 12)),
])
def test_resample_bitwise(dtype, nearest, src, dst):
    v = np.random.default_rng(7).standard_normal((3,) + src).astype(dtype)
    got = D.resample(torch.from_numpy(v).cuda(), dst, nearest).cpu().numpy()
    np.testing.assert_array_equal(got, P.resample(v, dst, nearest))


def test_scale_image_anisotropic_bitwise():
    v = np.random.default_rng(3).standard_normal((1, 20, 24, 18))
    sp = (0.8, 1.25, 2.0)
    got = D.scale_image(torch.from_numpy(v).cuda(), sp, (10, 12, 9)).cpu().numpy()
    np.testing.assert_array_equal(got, P.scale_image(v, sp, (10, 12, 9)))


@pytest.mark.parametrize("kw", [
    dict(levels=2, it_max=[25, 25]),
    dict(levels=3, it_max=[10, 10, 10], pad=1),
    dict(levels=2, it_max=[20, 15], redistribute=True),
    dict(levels=2, it_max=30, initial_guess=True, spacing=(1.0, 1.2, 0.9)),
    dict(levels=2, it_max=[20, 20], algorithm="greedy"),
    dict(levels=2, it_max=[20, 20], smoothing="sampled"),
])
def test_driver_fp64_matches_oracle(kw):
    kw = dict(kw)
    Jt, mask = ball_problem(34, 16, 7, 1.1)
    if kw.pop("initial_guess", False):
        kw["initial_guess"] = np.random.default_rng(5).normal(scale=0.05, size=(3,) + Jt.shape)
    got = D.displacement(Jt, mask=mask, precision="fp64", **kw)
    ref = P.displacement(Jt, mask=mask, **kw)
    assert got.shape == ref.shape == (3,) + Jt.shape
    assert np.max(np.abs(got - ref)) <= 1e-10


def test_driver_mixed_final_residual():
    Jt, mask = ball_problem(34, 16, 7, 1.1)
    got, stats = D.displacement(Jt, mask=mask, levels=2, it_max=[300, 1000], precision="mixed",
                                return_stats=True)
    ref = P.displacement(Jt, mask=mask, levels=2, it_max=[300, 1000], field_dtype=np.float32)
    from oracle.oracle import Oracle
    o = Oracle(4)
    r_got = masked_max(o.jacobian(got), Jt, mask)
    r_ref = masked_max(o.jacobian(ref), Jt, mask)
    assert len(stats) == 2
    assert abs(r_got - r_ref) <= 1e-4, (r_got, r_ref)


def test_driver_argument_errors():
    Jt, mask = ball_problem(12, 6, 3, 1.1)
    with pytest.raises(ValueError):
        D.displacement(Jt, mask=mask, levels=2, it_max=[5])
    with pytest.raises(ValueError):
        D.displacement(Jt, mask=mask[:-1])
    with pytest.raises(ValueError):
        D.displacement(Jt, mask=mask, algorithm="newton")


def test_driver_matching_matches_reference():
    """The wrapper with the matching solver at every level against the
    reference's volume_matching_3d run through the restated pyramid
    (tests/golden/matching_pyramid.npz; both solvers compute in FP32, fields
    agree to 2e-3 as for one level).  A device tensor gives the same field."""
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "matching_pyramid.npz"))
    kw = dict(levels=int(d["levels"]), it_max=[int(v) for v in d["it_max"]], spacing=tuple(d["spacing"]),
              algorithm="matching")
    got = D.displacement(d["Jt"], mask=d["mask"], **kw)
    assert got.shape == d["out"].shape
    assert np.max(np.abs(got - d["out"])) <= 2e-3
    dev = D.displacement(torch.from_numpy(d["Jt"]).cuda(), mask=torch.from_numpy(d["mask"]).cuda(), **kw)
    assert dev.dtype == torch.float64
    np.testing.assert_array_equal(dev.cpu().numpy(), got)
