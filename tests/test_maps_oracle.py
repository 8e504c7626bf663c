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


def _golden_maps():
    import os
    return dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "maps.npz")))


def test_restatement_matches_reference_functions():
    """The restatement against the reference's own map functions
    (disptools/displacements.py:486-668, executed by tests/golden/make_golden.py)."""
    g = _golden_maps()
    maps = [g[f"map{k}"] for k in range(4)]
    fields = [g[f"field{k}"] for k in range(3)]
    sp = tuple(g["spacing"])
    for eps, tag in ((1e-5, "1em05"), (0.3, "0p3")):
        np.testing.assert_array_equal(O.jacobian_to_volume_change(maps[0], eps), g[f"volume_change_{tag}"])
        np.testing.assert_allclose(O.average_jacobian(maps, eps), g[f"average_jacobian_{tag}"], rtol=1e-14)
        np.testing.assert_allclose(O.average_jacobian_from_displacements(fields, eps, sp),
                                   g[f"average_from_fields_{tag}"], rtol=1e-14)
