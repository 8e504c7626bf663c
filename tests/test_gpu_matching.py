"""The matching solver (volume_matching_3d) on the device against the
reference's own results (tests/golden/matching.npz, made from
src/VolumeMatching3D.c by tests/golden/make_golden.py).

Both compute in FP32; the reference sums the cost sequentially in float and
the device in FP64, so the step-control decisions can differ in the last
bits of a comparison: fields agree to 2e-3 (typically to float rounding) and
the final masked residuals to 1e-3."""
from __future__ import annotations

import os

import numpy as np
import pytest

import disptools_b200 as dt
from tests.helpers import ball_problem, masked_max

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def cases():
    d = np.load(os.path.join(HERE, "golden", "matching.npz"))
    count = len({name.split("_")[0] for name in d.files})
    return [tuple(d[f"m{k}_{n}"] for n in ("Jt", "mask", "field0", "spacing", "it_max", "out"))
            for k in range(count)]


def test_matching_matches_reference(cases, oracle):
    for Jt, m, f0, sp, it, ref in cases:
        out, st = dt.solve(Jt, m, f0, spacing=tuple(sp), algorithm="matching", it_max=int(it))
        assert st["iterations"] == int(it)
        assert np.max(np.abs(out - ref)) <= 2e-3
        r_ref = masked_max(oracle.jacobian(ref, tuple(sp)), Jt, m)
        r_out = masked_max(oracle.jacobian(out, tuple(sp)), Jt, m)
        assert abs(r_out - r_ref) <= 1e-3, (r_out, r_ref)


def test_matching_entry_points_agree(cases):
    """The extension, the reference-named C function and the Python API give
    the same field."""
    from disptools_b200 import _disptools
    from disptools_b200 import _native as N
    Jt, m, f0, sp, it, _ = cases[1]
    a, _ = dt.solve(Jt, m, f0, spacing=tuple(sp), algorithm="matching", it_max=int(it))
    b = np.ascontiguousarray(f0.copy())
    args = [9.99e-4, 0.2, 0.1, 0.4, 1.2, 0.5, 0.1, 1e-3, 10.0, 1e-6, 1e-9]
    _disptools.displacement(tuple(sp), Jt, m, *args, False, int(it), b, "matching", -1)
    c = np.ascontiguousarray(f0.copy())
    nz, ny, nx = Jt.shape
    N.lib.volume_matching_3d(nx, ny, nz, *map(float, sp), Jt.ctypes.data, m.ctypes.data, *args, False,
                             int(it), c.ctypes.data)
    assert not N.lib.disptools_has_error()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)


def test_matching_cost_decreases_and_stops():
    Jt, m = ball_problem(24, 12, 6, 0.9)
    _, s0 = dt.solve(Jt, m, algorithm="matching", it_max=0)
    out, s1 = dt.solve(Jt, m, algorithm="matching", it_max=25)
    assert s0["iterations"] == 0 and s1["iterations"] == 25
    assert s1["error"] < s0["error"]
    assert np.isfinite(out).all()
    # a loose epsilon stops the solver before it_max
    _, s2 = dt.solve(Jt, m, algorithm="matching", it_max=500, epsilon=0.05)
    assert s2["iterations"] < 500 and s2["max_error"] <= 0.05


def test_matching_device_entry_equals_host(cases):
    """dtb_volume_matching_device (through torch_ops.solve on float64
    tensors, on a side stream) gives the host entry's field bit for bit;
    float32 tensors are refused."""
    import torch

    from disptools_b200 import torch_ops
    Jt, m, f0, sp, it, _ = cases[3]
    a, sa = dt.solve(Jt, m, f0, spacing=tuple(sp), algorithm="matching", it_max=int(it))
    Jd, md = torch.from_numpy(Jt).cuda(), torch.from_numpy(m).cuda()
    fd = torch.from_numpy(f0.copy()).cuda()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        st = torch_ops.solve(Jd, md, fd, spacing=tuple(sp), algorithm="matching", it_max=int(it))
    torch.cuda.current_stream().wait_stream(side)
    np.testing.assert_array_equal(fd.cpu().numpy(), a)
    assert (st["iterations"], st["reason"]) == (sa["iterations"], sa["reason"])
    with pytest.raises(ValueError):
        torch_ops.solve(Jd.float(), md, fd.float(), spacing=tuple(sp), algorithm="matching", it_max=1)


def test_matching_profile_counts_kernels():
    """With profiling on, every gradient and cost launch of the matching
    solver is timed."""
    Jt, m = ball_problem(20, 10, 5, 1.1)
    dt.set_profiling(True)
    try:
        _, st = dt.solve(Jt, m, algorithm="matching", it_max=5)
        prof = dt.kernel_profile()
    finally:
        dt.set_profiling(False)
    assert st["iterations"] == 5
    g, c = prof["match_gradient"], prof["match_cost"]
    assert g[0] >= 5 and c[0] >= g[0] + 1
    assert g[1] > 0.0 and c[1] > 0.0
