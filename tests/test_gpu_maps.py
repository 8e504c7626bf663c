"""Jacobian-map utilities on the device against their CPU restatement
(oracle/maps.py), and against golden vectors made by the reference's own map
functions and regularise (tests/golden/maps.npz)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from disptools_b200 import io as fio
from disptools_b200 import maps as M
from oracle import maps as O

pytestmark = pytest.mark.gpu


def _maps(k, shape=(9, 11, 13), seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        J = rng.uniform(-0.2, 2.5, shape)
        J.flat[:4] = [0.0, 1e-6, 1.0, 2e9]
        out.append(J)
    return out


def test_volume_change_fp64_and_fp32():
    J = _maps(1)[0]
    J.flat[5] = np.nan
    got = M.jacobian_to_volume_change(J, 1e-5)
    ref = O.jacobian_to_volume_change(J, 1e-5)
    np.testing.assert_array_equal(got, ref)
    J32 = J.astype(np.float32)
    got32 = M.jacobian_to_volume_change(torch.from_numpy(J32).cuda(), 1e-5).cpu().numpy()
    np.testing.assert_array_equal(got32, O.jacobian_to_volume_change(J32, np.float32(1e-5)))


def test_average_jacobian_arrays_files_and_tensors(tmp_path):
    maps = _maps(4, seed=1)
    ref = O.average_jacobian(maps, 1e-5)
    np.testing.assert_allclose(M.average_jacobian(maps, 1e-5), ref, rtol=1e-14)
    for i, m in enumerate(maps):
        fio.write_vtk(tmp_path / f"j{i}.vtk", m)
    np.testing.assert_allclose(M.average_jacobian(str(tmp_path / "j*.vtk"), 1e-5), ref, rtol=1e-14)
    t = M.average_jacobian([torch.from_numpy(m).cuda() for m in maps], 1e-5)
    assert isinstance(t, torch.Tensor) and t.is_cuda
    np.testing.assert_allclose(t.cpu().numpy(), ref, rtol=1e-14)


def test_average_jacobian_from_displacements(tmp_path):
    rng = np.random.default_rng(2)
    fields = [rng.normal(scale=0.3, size=(3, 8, 9, 10)) for _ in range(3)]
    sp = (0.9, 1.1, 1.3)
    ref = O.average_jacobian_from_displacements(fields, 1e-5, sp)
    np.testing.assert_allclose(M.average_jacobian_from_displacements(fields, 1e-5, sp), ref,
                               rtol=1e-14)
    for i, f in enumerate(fields):
        fio.write_rvf(tmp_path / f"u{i}.rvf", f, sp)
    # spacings travel through the file as %f text and a float, like the reference
    sp_file = tuple(float(np.float32(v)) for v in sp)
    ref_file = O.average_jacobian_from_displacements(fields, 1e-5, sp_file)
    np.testing.assert_allclose(M.average_jacobian_from_displacements(str(tmp_path / "u*.rvf"), 1e-5),
                               ref_file, rtol=1e-14)


def test_map_argument_errors():
    with pytest.raises(ValueError):
        M.average_jacobian([], 1e-5)
    with pytest.raises(ValueError):
        M.average_jacobian([np.ones((3, 3, 3)), np.ones((3, 3, 4))])


def _golden_maps():
    import os
    return dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "maps.npz")))


def test_maps_match_reference_functions():
    """Device results against the reference's own functions
    (disptools/displacements.py:486-668) on the same inputs."""
    g = _golden_maps()
    maps = [g[f"map{k}"] for k in range(4)]
    fields = [g[f"field{k}"] for k in range(3)]
    sp = tuple(g["spacing"])
    for eps, tag in ((1e-5, "1em05"), (0.3, "0p3")):
        np.testing.assert_array_equal(M.jacobian_to_volume_change(maps[0], eps), g[f"volume_change_{tag}"])
        np.testing.assert_allclose(M.average_jacobian(maps, eps), g[f"average_jacobian_{tag}"], rtol=1e-14)
        np.testing.assert_allclose(M.average_jacobian_from_displacements(fields, eps, sp),
                                   g[f"average_from_fields_{tag}"], rtol=1e-14)


def test_regularise_matches_reference_with_nan():
    """dt.regularise against the reference's regularise (src/jacobian.c:29-55,
    through its Python wrapper): values below epsilon, -inf and -0.0 become
    epsilon; NaN and +inf stay."""
    import disptools_b200 as dt
    g = _golden_maps()
    got = dt.regularise(g["regularise_in"], 0.05)
    np.testing.assert_array_equal(got, g["regularise_out_0p05"])
    # the reference C library itself, on the same input
    from oracle.oracle import Reference
    if Reference.available("ref64"):
        np.testing.assert_array_equal(got, Reference("ref64").regularise(g["regularise_in"], 0.05))
