"""Failure detection and the auxiliary paths, without faulting the GPU:
an allocation refused by the memory limit, a TMA load that one tile skips
(its bounded wait runs out and the solve reports an error), non-finite
inputs, verbose output against the reference's own, determinism, and every
tiny shape against the oracle."""
from __future__ import annotations

import ctypes as C
import itertools
import os
import re

import numpy as np
import pytest

import disptools_b200 as dt
from disptools_b200 import _native as N
from tests.helpers import ball_problem

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def test_memory_limit_refuses_then_recovers():
    Jt, m = ball_problem(32, 16, 8, 1.1)
    good, _ = dt.solve(Jt, m, precision="fp64", it_max=10)
    N.check(N.lib.dtb_set_device_memory_limit(1 << 20))
    try:
        with pytest.raises(dt.DisptoolsError, match="memory"):
            dt.solve(Jt, m, precision="fp64", it_max=10)
    finally:
        N.check(N.lib.dtb_set_device_memory_limit(0))
    again, _ = dt.solve(Jt, m, precision="fp64", it_max=10)
    np.testing.assert_array_equal(good, again)


@pytest.mark.parametrize("algorithm,trial_kernel", [("gradient", "formed"), ("gradient", "release"),
                                                    ("greedy", "formed")])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_dropped_tma_load_is_reported_and_device_recovers(precision, algorithm, trial_kernel, monkeypatch):
    """The greedy trial also has element copies of the boundary values in
    flight when its wait runs out; they complete before the block leaves.
    The trial kernel without a plane barrier agrees on the fault after its
    plane loop and waits for the last load of each slot."""
    monkeypatch.setenv("DISPTOOLS_B200_TRIAL_KERNEL", trial_kernel)
    Jt, m = ball_problem(40, 20, 9, 1.1)
    good, sg = dt.solve(Jt, m, precision=precision, algorithm=algorithm, it_max=15)
    N.check(N.lib.dtb_test_drop_tma_load(0, 5, 1 << 12))
    try:
        with pytest.raises(dt.DisptoolsError, match="did not complete within its bound"):
            dt.solve(Jt, m, precision=precision, algorithm=algorithm, it_max=15)
    finally:
        N.check(N.lib.dtb_test_drop_tma_load(-1, -1, 0))
    again, sa = dt.solve(Jt, m, precision=precision, algorithm=algorithm, it_max=15)
    np.testing.assert_array_equal(good, again)
    assert sg["iterations"] == sa["iterations"]


def test_non_finite_initial_field_matches_oracle(oracle):
    Jt, m = ball_problem(12, 6, 3, 1.1)
    f0 = np.zeros((3, 12, 12, 12))
    f0[0, 6, 6, 6] = np.inf
    ref, so = oracle.solve("gradient", Jt, m, field=f0, it_max=20)
    out, st = dt.solve(Jt, m, f0, precision="fp64", it_max=20)
    assert st["reason"] == so.reason and st["iterations"] == so.iterations
    np.testing.assert_array_equal(np.isfinite(out), np.isfinite(ref))


def _reference_verbose_lines(Jt, m, capfd, **kw):
    path = os.path.join(REF_DIR, "libdisptools_ref64_verbose.so")
    if not os.path.exists(path):
        pytest.skip("verbose reference build not present (oracle/Makefile ref)")
    from oracle.oracle import Reference
    r = Reference("ref64_verbose")
    capfd.readouterr()
    r.solve("gradient", Jt, m, **kw)
    out = capfd.readouterr().out
    return [l for l in out.splitlines() if l.startswith(("Iteration", "Terminating", "Error not"))]


def test_verbose_output_matches_reference(capfd):
    Jt, m = ball_problem(24, 12, 6, 1.1)
    want = _reference_verbose_lines(Jt, m, capfd, it_max=300)
    prev = dt.set_verbose(True)
    try:
        capfd.readouterr()
        dt.solve(Jt, m, precision="fp64", it_max=300)
        got = capfd.readouterr().out.splitlines()
    finally:
        dt.set_verbose(prev)
    got = [l for l in got if l.startswith(("Iteration", "Terminating", "Error not"))]
    assert len(want) > 10 and got == want


def test_verbose_greedy_lines(capfd):
    Jt, m = ball_problem(16, 8, 4, 1.1)
    prev = dt.set_verbose(True)
    try:
        capfd.readouterr()
        _, st = dt.solve(Jt, m, precision="fp64", algorithm="greedy", it_max=30)
        out = capfd.readouterr().out.splitlines()
    finally:
        dt.set_verbose(prev)
    its = [l for l in out if l.startswith("Iteration")]
    assert its and all(re.match(r"Iteration +\d+:  total error \S+  max voxel error \S+  eta \S+$", l)
                       for l in its)
    assert st["trials"] == len(its)


def test_repeated_solves_are_bit_identical():
    from disptools_b200.synthetic import blob_problem
    Jt, m = blob_problem((48, 40, 56), blobs=4, seed=9)
    a, sa = dt.solve(Jt, m, precision="mixed", it_max=30)
    b, sb = dt.solve(Jt, m, precision="mixed", it_max=30)
    np.testing.assert_array_equal(a, b)
    assert sa["error"] == sb["error"] and sa["trials"] == sb["trials"]


def test_every_tiny_shape_jacobian_fp64(oracle):
    """All shapes with axes in 3..9 (343 volumes): the FP64 device Jacobian
    equals the oracle's."""
    rng = np.random.default_rng(0)
    for shape in itertools.product(range(3, 10), repeat=3):
        f = rng.normal(scale=0.3, size=(3,) + shape)
        sp = (1.0, 1.3, 0.7)
        np.testing.assert_allclose(dt.jacobian(f, sp), oracle.jacobian(f, sp), rtol=0, atol=1e-13)


@pytest.mark.parametrize("shape", [(3, 3, 3), (3, 9, 4), (9, 3, 5), (4, 5, 3), (9, 9, 9), (5, 7, 6)])
def test_tiny_shapes_solver_fp64(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    Jt = np.ascontiguousarray(1.0 + 0.05 * rng.standard_normal(shape))
    m = np.ascontiguousarray(rng.random(shape) < 0.5)
    for alg in ("gradient", "greedy"):
        ref, so = oracle.solve(alg, Jt, m, it_max=30)
        out, st = dt.solve(Jt, m, precision="fp64", algorithm=alg, it_max=30)
        assert st["iterations"] == so.iterations and st["reason"] == so.reason
        assert np.max(np.abs(out - ref)) <= 1e-10
