"""The NumPy extension mirrors the reference _disptools module
(python_c_extension/_disptools.c:532-540); argument errors are raised on the
host, before any device work."""
from __future__ import annotations

import numpy as np
import pytest

from disptools_b200 import _disptools

ARGS = dict(epsilon=9.99e-4, tolerance=0.2, eta=0.1, eta_max=0.4, alpha=1.2, beta=0.5,
            gamma=0.1, delta=1e-3, zeta=10.0, theta=1e-6, iota=1e-9, strict=False, it_max=10)


def call(J, mask, field, algorithm="gradient", gpu_id=-1, **over):
    a = {**ARGS, **over}
    return _disptools.displacement((1.0, 1.0, 1.0), J, mask, a["epsilon"], a["tolerance"], a["eta"],
                                   a["eta_max"], a["alpha"], a["beta"], a["gamma"], a["delta"],
                                   a["zeta"], a["theta"], a["iota"], a["strict"], a["it_max"], field,
                                   algorithm, gpu_id)


def test_method_table():
    for name in ("error_out", "get_float_type_size", "regularise", "shape_descriptor", "jacobian",
                 "displacement"):
        assert callable(getattr(_disptools, name))
    assert _disptools.get_float_type_size() == 64
    with pytest.raises(NotImplementedError):
        _disptools.shape_descriptor(np.zeros((3, 3, 3)), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "cubeness")


def test_displacement_argument_errors():
    J = np.ones((5, 5, 5))
    m = np.ones((5, 5, 5), bool)
    f = np.zeros((3, 5, 5, 5))
    with pytest.raises(ValueError, match="Invalid algorithm"):
        call(J, m, f, algorithm="bogus")
    with pytest.raises(RuntimeError, match="at least 2 voxels"):  # matching: host-side check
        call(np.ones((1, 5, 5)), np.ones((1, 5, 5), bool), np.zeros((3, 1, 5, 5)), algorithm="matching")
    with pytest.raises(TypeError):
        call(J.astype(np.float32), m, f)
    with pytest.raises(TypeError):
        call(J, m.astype(np.uint8), f)
    with pytest.raises(ValueError):
        call(J, m, np.zeros((3, 5, 5, 4)))
    with pytest.raises(ValueError):
        call(J, np.ones((5, 5, 4), bool), f)
    with pytest.raises(ValueError):
        call(J, m, np.asfortranarray(np.zeros((3, 5, 5, 5))))
    with pytest.raises(ValueError):
        call(J, m, f, it_max=-1)
    with pytest.raises(TypeError):
        _disptools.displacement((1.0, 1.0, 1.0), J, m)


def test_jacobian_argument_errors():
    with pytest.raises(ValueError):
        _disptools.jacobian((1.0, 1.0), np.zeros((3, 4, 4, 4)), np.zeros((4, 4, 4)))
    with pytest.raises(ValueError):
        _disptools.jacobian((1.0, 1.0, 1.0), np.zeros((3, 4, 4, 5)), np.zeros((4, 4, 4)))
    with pytest.raises(TypeError):
        _disptools.jacobian((1.0, 1.0, 1.0), np.zeros((3, 4, 4, 4), np.float32), np.zeros((4, 4, 4)))


def test_error_out():
    with pytest.raises(Exception, match="something bad happened"):
        _disptools.error_out()
