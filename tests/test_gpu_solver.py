"""Solver parity against the FP64 oracle (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import disptools_b200 as dt
from tests.helpers import ball_problem, masked_max

pytestmark = pytest.mark.gpu


def _golden_case(golden, case):
    k = case["name"]
    s = golden["solver"]
    return s[f"{k}_Jt"], s[f"{k}_mask"], s[f"{k}_field0"], s[f"{k}_out"]


def test_golden_cases_fp64(golden):
    for case in golden["cases"]["cases"]:
        Jt, mask, f0, ref = _golden_case(golden, case)
        out, st = dt.solve(Jt, mask, f0, spacing=tuple(case["spacing"]), algorithm=case["algorithm"],
                           precision="fp64", **case["params"])
        assert np.max(np.abs(out - ref)) <= 1e-10, (case, st)


def test_golden_cases_mixed(golden, oracle):
    for case in golden["cases"]["cases"]:
        Jt, mask, f0, ref = _golden_case(golden, case)
        sp = tuple(case["spacing"])
        out, st = dt.solve(Jt, mask, f0, spacing=sp, algorithm=case["algorithm"], precision="mixed",
                           **case["params"])
        r_ref = masked_max(oracle.jacobian(ref, sp), Jt, mask)
        r_out = masked_max(oracle.jacobian(out, sp), Jt, mask)
        assert abs(r_out - r_ref) <= 1e-4, (case["name"], r_out, r_ref, st)


def test_config1_drop_in(golden, oracle):
    """Config 1 through the reference-named entry point and the extension."""
    from disptools_b200 import _disptools
    Jt, mask = ball_problem(40, 20, 10)
    c1 = golden["cases"]["config1"]
    args = [9.99e-4, 0.2, 0.1, 0.4, 1.2, 0.5, 0.1, 1e-3, 10.0, 1e-6, 1e-9, False, 1000]
    dt.set_default_precision("fp64")
    try:
        f = np.zeros((3, 40, 40, 40))
        _disptools.displacement((1.0, 1.0, 1.0), Jt, mask, *args, f, "gradient", 0)
    finally:
        dt.set_default_precision("mixed")
    assert masked_max(oracle.jacobian(f), Jt, mask) == pytest.approx(c1["masked_max"], rel=1e-9)
    np.testing.assert_allclose(f[:, 20, 20, :], np.array(c1["field_line"]), atol=1e-12)
    f32 = np.zeros((3, 40, 40, 40))
    _disptools.displacement((1.0, 1.0, 1.0), Jt, mask, *args, f32, "gradient", 0)
    assert abs(masked_max(oracle.jacobian(f32), Jt, mask) - c1["masked_max"]) <= 1e-4


def test_config1_stats_fp64_match_oracle(oracle):
    Jt, mask = ball_problem(40, 20, 10)
    ref, so = oracle.solve("gradient", Jt, mask, it_max=1000)
    out, st = dt.solve(Jt, mask, precision="fp64", it_max=1000)
    assert st["iterations"] == so.iterations == 123
    assert st["trials"] == so.trials
    assert st["reason"] == so.reason
    assert st["max_error"] == pytest.approx(so.max_error, rel=1e-12)
    assert st["error"] == pytest.approx(so.error, rel=1e-12)
    assert np.max(np.abs(out - ref)) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("algorithm", ["gradient", "greedy"])
def test_batched_equals_single(precision, algorithm):
    rng = np.random.default_rng(11)
    vols = []
    for n in [(12, 17, 9), (20, 20, 20), (7, 33, 15)]:
        Jt = 1.0 + 0.1 * rng.standard_normal(n)
        mask = rng.random(n) < 0.3
        vols.append((np.ascontiguousarray(Jt), np.ascontiguousarray(mask)))
    single = [dt.solve(J, m, algorithm=algorithm, precision=precision, it_max=40) for J, m in vols]
    batch = dt.solve_batched(vols, algorithm=algorithm, precision=precision, it_max=40)
    for (a, sa), (b, sb) in zip(single, batch):
        np.testing.assert_array_equal(a, b)
        assert sa["iterations"] == sb["iterations"] and sa["trials"] == sb["trials"]


EDGE_CASES = {
    "minimal_3": dict(shape=(3, 3, 3)),
    "thin_axis": dict(shape=(3, 17, 12)),
    "empty_mask": dict(shape=(10, 11, 12), empty=True),
    "it_max_0": dict(shape=(10, 10, 10), it_max=0),
    "it_max_1": dict(shape=(10, 10, 10), it_max=1),
    "strict": dict(shape=(14, 12, 10), strict=True),
    "nan_target": dict(shape=(10, 10, 10), nan=True),
    "anisotropic": dict(shape=(11, 13, 9), spacing=(0.5, 1.5, 2.5)),
}


@pytest.mark.parametrize("name", sorted(EDGE_CASES))
@pytest.mark.parametrize("algorithm", ["gradient", "greedy"])
def test_edge_cases_fp64_vs_oracle(oracle, name, algorithm):
    c = EDGE_CASES[name]
    shape = c["shape"]
    rng = np.random.default_rng(len(name))
    Jt = np.ascontiguousarray(1.0 + 0.08 * rng.standard_normal(shape))
    mask = np.zeros(shape, bool) if c.get("empty") else np.ascontiguousarray(rng.random(shape) < 0.5)
    if c.get("nan"):
        Jt[shape[0] // 2, shape[1] // 2, shape[2] // 2] = np.nan
    f0 = rng.normal(scale=0.01, size=(3,) + shape)
    sp = c.get("spacing", (1.0, 1.0, 1.0))
    kw = dict(it_max=c.get("it_max", 60), strict=c.get("strict", False))
    ref, so = oracle.solve(algorithm, Jt, mask, field=f0, spacing=sp, **kw)
    out, st = dt.solve(Jt, mask, f0, spacing=sp, algorithm=algorithm, precision="fp64", **kw)
    assert st["reason"] == so.reason and st["iterations"] == so.iterations, (st, so)
    assert np.max(np.abs(out - ref)) <= 1e-10


@pytest.mark.parametrize("trial_kernel", ["formed", "release"])
@pytest.mark.parametrize("name", sorted(EDGE_CASES))
def test_edge_cases_fp64_both_trial_kernels(oracle, monkeypatch, name, trial_kernel):
    """The gradient method's edge cases through each trial kernel, forced."""
    monkeypatch.setenv("DISPTOOLS_B200_TRIAL_KERNEL", trial_kernel)
    test_edge_cases_fp64_vs_oracle(oracle, name, "gradient")
    assert dt.tile_config()["trial_kernel"] == trial_kernel


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_equals_single_release_kernel(monkeypatch, precision):
    monkeypatch.setenv("DISPTOOLS_B200_TRIAL_KERNEL", "release")
    test_batched_equals_single(precision, "gradient")


@pytest.mark.parametrize("boundary", ["zero", "negative_zero", "one_voxel"])
def test_greedy_boundary_values_fp64_vs_oracle(oracle, boundary):
    """The greedy trial skips copying the new buffer's boundary values when
    they are all +0: an initial field that is zero on the boundary (the
    copies skipped in both buffers), -0.0 there (bitwise not +0: copied), or
    zero but for one boundary voxel (copied while buffer 0 is the new
    buffer).  Each must equal the oracle bit for bit."""
    shape = (37, 45, 70)
    rng = np.random.default_rng(23)
    Jt = np.ascontiguousarray(1.0 + 0.08 * rng.standard_normal(shape))
    mask = np.ascontiguousarray(rng.random(shape) < 0.5)
    f0 = rng.normal(scale=0.02, size=(3,) + shape)
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    f0[:, ~inner] = -0.0 if boundary == "negative_zero" else 0.0
    if boundary == "one_voxel":
        f0[1, 0, 20, 30] = 0.05
    ref, so = oracle.solve("greedy", Jt, mask, field=f0, it_max=25)
    out, st = dt.solve(Jt, mask, f0, algorithm="greedy", precision="fp64", it_max=25)
    assert st["reason"] == so.reason and st["iterations"] == so.iterations, (st, so)
    assert st["trials"] == so.trials
    assert np.max(np.abs(out - ref)) <= 1e-12


@pytest.mark.parametrize("shape", [(37, 45, 70), (70, 18, 33), (9, 40, 131)])
def test_greedy_multi_tile_fp64_vs_oracle(oracle, shape):
    """Greedy trials over several tiles along every axis, x extents that end
    inside a 16-byte chunk, anisotropic spacing: bit-level agreement."""
    rng = np.random.default_rng(sum(shape))
    Jt = np.ascontiguousarray(1.0 + 0.08 * rng.standard_normal(shape))
    mask = np.ascontiguousarray(rng.random(shape) < 0.5)
    f0 = rng.normal(scale=0.02, size=(3,) + shape)
    sp = (0.9, 1.1, 1.3)
    ref, so = oracle.solve("greedy", Jt, mask, field=f0, spacing=sp, it_max=25)
    out, st = dt.solve(Jt, mask, f0, spacing=sp, algorithm="greedy", precision="fp64", it_max=25)
    assert st["reason"] == so.reason and st["iterations"] == so.iterations, (st, so)
    assert st["trials"] == so.trials
    assert np.max(np.abs(out - ref)) <= 1e-12


def test_greedy_mixed_tracks_fp64():
    shape = (37, 45, 70)
    rng = np.random.default_rng(5)
    Jt = np.ascontiguousarray(1.0 + 0.08 * rng.standard_normal(shape))
    mask = np.ascontiguousarray(rng.random(shape) < 0.5)
    f64, s64 = dt.solve(Jt, mask, algorithm="greedy", precision="fp64", it_max=25)
    f32, s32 = dt.solve(Jt, mask, algorithm="greedy", precision="mixed", it_max=25)
    assert s32["iterations"] == s64["iterations"]
    assert np.max(np.abs(f32 - f64)) <= 1e-4
    assert s32["error"] == pytest.approx(s64["error"], rel=1e-3)


def test_device_tensor_solve_matches_host():
    import torch
    from disptools_b200 import torch_ops
    Jt, mask = ball_problem(24, 12, 6, 0.9)
    host, sh = dt.solve(Jt, mask, precision="mixed", it_max=100)
    f = torch.zeros((3, 24, 24, 24), dtype=torch.float32, device="cuda")
    st = torch_ops.solve(torch.from_numpy(Jt).float().cuda(), torch.from_numpy(mask).cuda(), f,
                         it_max=100)
    assert st["iterations"] == sh["iterations"]
    np.testing.assert_allclose(f.cpu().numpy(), host, atol=1e-7)


def test_full_size_256_fp64_first_iterations(oracle):
    """Config-2 inputs at full size: a few FP64 iterations against the oracle."""
    from disptools_b200.synthetic import blob_problem
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    ref, so = oracle.solve("gradient", Jt, mask, it_max=3)
    out, st = dt.solve(Jt, mask, precision="fp64", it_max=3)
    assert st["trials"] == so.trials and st["reason"] == so.reason
    assert st["error"] == pytest.approx(so.error, rel=1e-12)
    assert np.max(np.abs(out - ref)) <= 1e-10


def test_full_size_256_fp64_greedy_first_iterations(oracle):
    """Config-2 inputs at full size, greedy method: a few FP64 iterations
    against the oracle (every tile, both field buffers, the error maps)."""
    from disptools_b200.synthetic import blob_problem
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    ref, so = oracle.solve("greedy", Jt, mask, it_max=4)
    out, st = dt.solve(Jt, mask, algorithm="greedy", precision="fp64", it_max=4)
    assert st["iterations"] == so.iterations and st["trials"] == so.trials and st["reason"] == so.reason
    assert st["error"] == pytest.approx(so.error, rel=1e-12)
    assert np.max(np.abs(out - ref)) <= 1e-12


def test_full_size_256_fp64_matches_reference_at_it_max_100(oracle):
    """The headline workload (config 2 at 256^3, it_max 100) against the
    reference C library built with FP64 FLOATING, solving the same volume to
    the same it_max: the FP64 device path returns the reference's field
    (1e-10) after the same number of iterations.  (The mixed path's field
    differs by then: before convergence its accept/reject sequence drifts from
    the FP64 one, see the converged comparison below.)"""
    from disptools_b200.synthetic import blob_problem
    from oracle.oracle import Reference
    IT = 100
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    if Reference.available("ref64_verbose"):
        ref, _, its_ref = Reference("ref64_verbose").solve_logged("gradient", Jt, mask, it_max=IT)
    else:  # the restatement, pinned to the reference on the golden vectors
        ref, so = oracle.solve("gradient", Jt, mask, it_max=IT)
        its_ref = so.iterations - 1 if so.reason == "it_max" else so.iterations
    out64, st64 = dt.solve(Jt, mask, precision="fp64", it_max=IT)
    its64 = st64["iterations"] - 1 if st64["reason"] == "it_max" else st64["iterations"]
    assert its64 == its_ref, (st64, its_ref)
    assert np.max(np.abs(out64 - ref)) <= 1e-10


def _config2_reference():
    import json
    import os
    p = os.path.join(os.path.dirname(__file__), "golden", "config2_converged.json")
    if not os.path.exists(p):
        pytest.skip("tests/golden/config2_converged.json not generated")
    return json.load(open(p))


def test_full_size_256_converged_mixed_within_1e4_of_reference(oracle):
    """The accuracy rule at the headline size: config 2 solved to the
    solver's own termination (default parameters, it_max 50000), the mixed
    path's final masked max |J - J_t| (recomputed in FP64) within 1e-4 of
    the reference C library's (FP64), whose converged run is summarised in
    tests/golden/config2_converged.json (made by make_golden.py --config2:
    thousands of iterations, too long for a test on the host).  The FP64
    device path to termination gives the reference's residual to 1e-9."""
    from disptools_b200.synthetic import blob_problem
    ref = _config2_reference()
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    out32, st32 = dt.solve(Jt, mask, precision="mixed", it_max=50000)
    r32 = masked_max(oracle.jacobian(out32), Jt, mask)
    assert abs(r32 - ref["masked_max"]) <= 1e-4, (r32, ref["masked_max"], st32)
    out64, st64 = dt.solve(Jt, mask, precision="fp64", it_max=50000)
    r64 = masked_max(oracle.jacobian(out64), Jt, mask)
    assert abs(r64 - ref["masked_max"]) <= 1e-9, (r64, ref["masked_max"], st64)
    assert st64["iterations"] == ref["iterations"], (st64, ref["iterations"])
    # both stop by the improvement rule ("Error not decreasing, terminating.")
    assert st64["reason"] == st32["reason"] == "improvement < theta"
    assert ref["stop_line"] == "Error not decreasing, terminating."


def test_full_size_256_mixed_properties(oracle):
    """Config-2 inputs at full size, mixed precision: the reported error of the
    returned field matches an FP64 recomputation, and it decreased."""
    from disptools_b200.synthetic import blob_problem
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    out, st = dt.solve(Jt, mask, precision="mixed", it_max=25)
    J = oracle.jacobian(out)
    assert abs(masked_max(J, Jt, mask) - st["max_error"]) <= 1e-5
    tot, mx, _ = oracle.compute_error(Jt, J, mask, 0.2)
    assert tot == pytest.approx(st["error"], rel=1e-4)
    _, s0 = dt.solve(Jt, mask, precision="mixed", it_max=0)
    assert st["error"] < s0["error"]


def test_config4_batched_vs_oracle(oracle):
    """Config-4 shaped batch (ellipsoid targets, one size per volume), scaled
    down so the oracle finishes in seconds: the batched FP64 solve equals the
    oracle's solve of each volume, the batched mixed solve meets the residual
    rule."""
    from disptools_b200.synthetic import batch_sizes, ellipsoid_problem
    sizes = batch_sizes(6, low=16, high=40, seed=4)
    vols = [ellipsoid_problem(s, seed=i) for i, s in enumerate(sizes)]
    res64 = dt.solve_batched(vols, precision="fp64", it_max=80)
    for (Jt, mask), (f64, s64) in zip(vols, res64):
        ref, so = oracle.solve("gradient", Jt, mask, it_max=80)
        assert s64["iterations"] == so.iterations and s64["reason"] == so.reason
        assert np.max(np.abs(f64 - ref)) <= 1e-10
    # final residuals of full solves (the residual rule holds at the end of
    # a solve, not along the way)
    res32 = dt.solve_batched(vols, precision="mixed", it_max=1000)
    for (Jt, mask), (f32, _) in zip(vols, res32):
        ref, _ = oracle.solve("gradient", Jt, mask, it_max=1000)
        r_ref = masked_max(oracle.jacobian(ref), Jt, mask)
        r_32 = masked_max(oracle.jacobian(f32), Jt, mask)
        assert abs(r_32 - r_ref) <= 1e-4, (r_32, r_ref)


def test_config4_batched_large_properties(oracle):
    """Twelve volumes with axes in [48, 128] in one mixed batched solve: the
    reported masked maximum of every volume matches an FP64 recomputation
    and no volume's error grew."""
    from disptools_b200.synthetic import batch_sizes, ellipsoid_problem
    sizes = batch_sizes(12, low=48, high=128, seed=5)
    vols = [ellipsoid_problem(s, seed=100 + i) for i, s in enumerate(sizes)]
    res = dt.solve_batched(vols, precision="mixed", it_max=12)
    res0 = dt.solve_batched(vols, precision="mixed", it_max=0)
    for (Jt, mask), (f, st), (_, s0) in zip(vols, res, res0):
        J = oracle.jacobian(f)
        assert abs(masked_max(J, Jt, mask) - st["max_error"]) <= 1e-5
        assert st["error"] <= s0["error"]


def test_release_device_memory_then_solve_again():
    """Freeing the cached device memory between solves changes no result."""
    Jt, mask = ball_problem(20, 10, 5, 0.9)
    a, sa = dt.solve(Jt, mask, precision="mixed", it_max=30)
    dt.release_device_memory()
    b, sb = dt.solve(Jt, mask, precision="mixed", it_max=30)
    dt.release_device_memory()
    c, sc = dt.solve_batched([(Jt, mask)], precision="fp64", it_max=30)[0]
    d, sd = dt.solve(Jt, mask, precision="fp64", it_max=30)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(c, d)
    assert sa["iterations"] == sb["iterations"] and sc["iterations"] == sd["iterations"]


TILE_CANDIDATES = [
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 16, "bz": 32, "trial_kernel": "formed"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 8, "bz": 32, "trial_kernel": "formed"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 16, "bz": 16, "trial_kernel": "formed"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 16, "bz": 64, "trial_kernel": "formed"},
    {"tile_x": 32, "trial_threads_y": 8, "gradient_threads_y": 16, "bz": 32, "trial_kernel": "formed"},
    {"tile_x": 64, "trial_threads_y": 16, "gradient_threads_y": 8, "bz": 32, "trial_kernel": "formed"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 16, "bz": 32, "trial_kernel": "release"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 8, "bz": 16, "trial_kernel": "release"},
    {"tile_x": 32, "trial_threads_y": 16, "gradient_threads_y": 16, "bz": 29, "trial_kernel": "release"},
    {"tile_x": 32, "trial_threads_y": 8, "gradient_threads_y": 16, "bz": 32, "trial_kernel": "release"},
    {"tile_x": 64, "trial_threads_y": 16, "gradient_threads_y": 8, "bz": 32, "trial_kernel": "release"},
]
ENV_OF = (("TILE_X", "tile_x"), ("TRIAL_THREADS_Y", "trial_threads_y"), ("THREADS_Y", "gradient_threads_y"),
          ("BZ", "bz"), ("TRIAL_KERNEL", "trial_kernel"))


def _is_candidate(cfg) -> bool:
    """A shape the autotuner may choose: a listed x-y shape with the
    formed-plane trial kernel, and a z depth that is listed or wave-filled
    (12..64 planes)."""
    key = lambda c: (c["tile_x"], c["trial_threads_y"], c["gradient_threads_y"], c["trial_kernel"])  # noqa: E731
    return (cfg["trial_kernel"] == "formed" and any(key(c) == key(cfg) for c in TILE_CANDIDATES)
            and 12 <= cfg["bz"] <= 64)


def test_autotuned_shapes(oracle, monkeypatch):
    """A volume large enough for the autotuner (2.3 M voxels): the chosen
    shapes are candidates; the FP64 solve with the tuned shapes equals the
    oracle's; forcing the tuned shapes through the environment reproduces
    the tuned mixed solve bit for bit."""
    from disptools_b200.synthetic import blob_problem
    Jt, mask = blob_problem((112, 128, 160), blobs=6, seed=3)
    prev = dt.set_autotune(True)
    try:
        out64, _ = dt.solve(Jt, mask, precision="fp64", it_max=3)
        cfg64 = dt.tile_config()
        out32, _ = dt.solve(Jt, mask, precision="mixed", it_max=6)
        cfg32 = dt.tile_config()
    finally:
        dt.set_autotune(prev)
    assert _is_candidate(cfg64) and cfg64["tile_x"] == 32
    assert _is_candidate(cfg32)
    ref, _ = oracle.solve("gradient", Jt, mask, it_max=3)
    assert np.max(np.abs(out64 - ref)) <= 1e-10
    for k, v in ENV_OF:
        monkeypatch.setenv("DISPTOOLS_B200_" + k, str(cfg32[v]))
    again, _ = dt.solve(Jt, mask, precision="mixed", it_max=6)
    assert dt.tile_config() == cfg32
    np.testing.assert_array_equal(out32, again)


@pytest.mark.parametrize("shape", TILE_CANDIDATES)
def test_every_tile_shape_fp64_matches_oracle(oracle, monkeypatch, shape):
    """Each candidate shape (forced through the environment) gives the
    oracle's FP64 result on a volume with ragged tiles in every axis."""
    if shape["tile_x"] == 64:
        pytest.skip("64-wide tiles are FP32 only")
    for k, v in ENV_OF:
        monkeypatch.setenv("DISPTOOLS_B200_" + k, str(shape[v]))
    Jt, mask = ball_problem(45, 20, 9, 0.9)
    out, st = dt.solve(Jt, mask, precision="fp64", it_max=40)
    assert dt.tile_config() == shape
    ref, so = oracle.solve("gradient", Jt, mask, it_max=40)
    assert st["iterations"] == so.iterations
    assert np.max(np.abs(out - ref)) <= 1e-10


@pytest.mark.parametrize("shape", TILE_CANDIDATES)
def test_every_tile_shape_mixed_residual(oracle, monkeypatch, shape):
    for k, v in ENV_OF:
        monkeypatch.setenv("DISPTOOLS_B200_" + k, str(shape[v]))
    Jt, mask = ball_problem(45, 20, 9, 0.9)
    out, st = dt.solve(Jt, mask, precision="mixed", it_max=1000)
    assert dt.tile_config() == shape
    ref, _ = oracle.solve("gradient", Jt, mask, it_max=1000)
    r_ref = masked_max(oracle.jacobian(ref), Jt, mask)
    assert abs(masked_max(oracle.jacobian(out), Jt, mask) - r_ref) <= 1e-4


def test_batched_inplace_equals_copying():
    rng = np.random.default_rng(12)
    vols = []
    for n in [(10, 12, 9), (16, 8, 11)]:
        Jt = np.ascontiguousarray(1.0 + 0.1 * rng.standard_normal(n))
        mask = np.ascontiguousarray(rng.random(n) < 0.4)
        vols.append((Jt, mask, np.zeros((3,) + n)))
    copied = dt.solve_batched(vols, it_max=20)
    res = dt.solve_batched(vols, it_max=20, inplace=True)
    for (a, sa), (b, sb), v in zip(copied, res, vols):
        assert b is v[2]
        np.testing.assert_array_equal(a, b)
        assert sa["iterations"] == sb["iterations"]
    with pytest.raises(ValueError):
        dt.solve_batched([(vols[0][0], vols[0][1], np.zeros((3, 10, 12, 9), np.float32))], inplace=True)
