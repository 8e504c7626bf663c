"""CPU restatement of the reference's Jacobian-map utilities (test
infrastructure: the checker of disptools_b200.maps).

Follows disptools/displacements.py line by line on NumPy arrays; the
Jacobians of fields come from the C oracle (dt_oracle.c), which is pinned
to the reference build.  Pinned to the reference's own map functions by the
golden vectors of tests/golden/maps.npz (tests/test_maps_oracle.py).  The reference's NaN handling differs in one
place: its volume-change map leaves NaN voxels uninitialised (np.empty,
:658), which this restatement and the device code both return as NaN.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle


def jacobian_to_volume_change(jacobian, epsilon=1e-5):
    """disptools/displacements.py:651-668."""
    data = np.array(jacobian, copy=True)
    processed = np.full(data.shape, np.nan, dtype=data.dtype)
    ind_expa = data >= 1.0
    ind_comp = data < 1.0
    ind_sing = data <= epsilon
    data[ind_sing] = epsilon
    processed[ind_expa] = data[ind_expa] - 1.0
    processed[ind_comp] = 1.0 - (1.0 / data[ind_comp])
    return processed


def average_jacobian(maps, epsilon=1e-5):
    """disptools/displacements.py:603-625; sitk.Threshold(lower=epsilon,
    upper=1e9, outsideValue=epsilon) keeps [epsilon, 1e9]."""
    total = None
    n = 0
    for m in maps:
        j = np.asarray(m, dtype=np.float64)
        j = np.where((j >= epsilon) & (j <= 1e9), j, epsilon)
        if total is None:
            total = np.zeros(j.shape, dtype=j.dtype)
        total += np.log(j)
        n += 1
    return np.exp(1.0 / n * total)


def average_jacobian_from_displacements(fields, epsilon=1e-5, spacing=(1.0, 1.0, 1.0)):
    """disptools/displacements.py:525-568: J = jacobian(field), regularise
    (src/jacobian.c:29-55), geometric mean."""
    o = Oracle(4)
    total = None
    n = 0
    for f in fields:
        J = o.jacobian(np.asarray(f, dtype=np.float64), spacing)
        J = np.where(J < epsilon, epsilon, J)
        if total is None:
            total = np.zeros(J.shape)
        total += np.log(J)
        n += 1
    return np.exp(1.0 / n * total)
