"""The CPU restatement of the Jacobian-map utilities (oracle/maps.py)
against known answers."""
from __future__ import annotations

import numpy as np

from oracle import maps as O


def test_volume_change_known_values():
    J = np.array([2.0, 1.0, 0.5, 0.25, 0.0, -1.0, 1e-6])
    vc = O.jacobian_to_volume_change(J, 1e-5)
    sing = 1.0 - 1.0 / 1e-5
    np.testing.assert_array_equal(vc, [1.0, 0.0, -1.0, -3.0, sing, sing, sing])


def test_average_jacobian_known_values():
    a = np.full((2, 2, 2), 4.0)
    b = np.full((2, 2, 2), 0.25)
    np.testing.assert_allclose(O.average_jacobian([a, b]), 1.0, rtol=1e-15)
    np.testing.assert_allclose(O.average_jacobian([a, a, a]), 4.0, rtol=1e-15)
    # thresholding: values outside [eps, 1e9] count as eps
    c = np.array([[[2e9, -1.0]]])
    np.testing.assert_allclose(O.average_jacobian([c], 1e-3), 1e-3, rtol=1e-15)


def test_average_jacobian_from_zero_displacements():
    f = np.zeros((3, 4, 5, 6))
    np.testing.assert_array_equal(O.average_jacobian_from_displacements([f, f]), 1.0)
