"""Jacobian kernels against the oracle and the golden vectors (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import disptools_b200 as dt

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def test_fp64_golden_vectors_bit_exact(golden):
    g = golden["jacobian"]
    np.testing.assert_array_equal(dt.jacobian(g["sin10_field"]), g["sin10_J"])
    np.testing.assert_array_equal(dt.jacobian(g["i2_field"], (2.0, 3.0, 4.0)), g["i2_J"])
    for k in range(4):
        f, sp = g[f"rand{k}_field"], tuple(g[f"rand{k}_spacing"])
        assert rel_err(dt.jacobian(f, sp), g[f"rand{k}_J"]) <= 1e-12


@pytest.mark.parametrize("shape", [(3, 3, 3), (3, 40, 5), (9, 33, 70), (64, 64, 64),
                                   (5, 130, 17), (37, 8, 31), (4, 4, 200)])
def test_fp64_shapes_vs_oracle(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.normal(scale=0.2, size=(3,) + shape)
    sp = tuple(rng.uniform(0.5, 2.0, 3))
    assert rel_err(dt.jacobian(f, sp), oracle.jacobian(f, sp)) <= 1e-12


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("order", [4, 2])
def test_device_entry_fp32_and_fp64(oracle, oracle_pd2, order):
    torch = _torch()
    from disptools_b200 import torch_ops
    o = oracle if order == 4 else oracle_pd2
    rng = np.random.default_rng(3)
    f = rng.normal(scale=0.2, size=(3, 21, 34, 45))
    sp = (0.9, 1.2, 1.05)
    ref = o.jacobian(f, sp)
    J64 = torch_ops.jacobian_raw(torch.from_numpy(f).cuda(), sp, order).cpu().numpy()
    assert rel_err(J64, ref) <= 1e-12
    J32 = torch_ops.jacobian_raw(torch.from_numpy(f).float().cuda(), sp, order).cpu().numpy()
    assert rel_err(J32.astype(np.float64), ref) <= 2e-5


@pytest.mark.parametrize("shape", [(37, 45, 68), (70, 18, 36), (3, 3, 4), (33, 17, 132), (5, 40, 8)])
def test_device_entry_tma_layouts(oracle, shape):
    """Rows a multiple of 16 bytes long take the TMA kernel: several tiles
    along every axis, partial tiles, thin volumes; FP64 to the last bits."""
    torch = _torch()
    from disptools_b200 import torch_ops
    rng = np.random.default_rng(sum(shape))
    f = rng.normal(scale=0.2, size=(3,) + shape)
    sp = tuple(rng.uniform(0.5, 2.0, 3))
    ref = oracle.jacobian(f, sp)
    J64 = torch_ops.jacobian_raw(torch.from_numpy(f).cuda(), sp).cpu().numpy()
    assert rel_err(J64, ref) <= 1e-12
    J32 = torch_ops.jacobian_raw(torch.from_numpy(f).float().cuda(), sp).cpu().numpy()
    assert rel_err(J32.astype(np.float64), ref) <= 2e-5


def test_device_entry_unaligned_field_takes_plain_kernel(oracle):
    """A field that starts off a 16-byte boundary goes to the plain-load
    kernel and gives the same map."""
    torch = _torch()
    from disptools_b200 import torch_ops
    shape = (9, 20, 24)
    rng = np.random.default_rng(7)
    f = rng.normal(scale=0.2, size=(3,) + shape)
    ref = oracle.jacobian(f)
    n = f.size
    buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(f.ravel()).cuda()
    view = buf[1:].view((3,) + shape)  # 8 bytes past the allocation's start
    assert view.data_ptr() % 16 == 8
    J = torch_ops.jacobian_raw(view).cpu().numpy()
    assert rel_err(J, ref) <= 1e-12
    np.testing.assert_array_equal(J, torch_ops.jacobian_raw(view.clone()).cpu().numpy())


def test_full_size_256_vs_oracle(oracle):
    torch = _torch()
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    f = smooth_field((256, 256, 256), sigma=6.0, max_disp=3.0, seed=5)
    ref = oracle.jacobian(f)
    J64 = torch_ops.jacobian_raw(torch.from_numpy(f).cuda()).cpu().numpy()
    assert rel_err(J64, ref) <= 1e-12
    J32 = torch_ops.jacobian_raw(torch.from_numpy(f).float().cuda()).cpu().numpy()
    assert rel_err(J32.astype(np.float64), ref) <= 1e-4


def test_regularise():
    rng = np.random.default_rng(0)
    J = rng.random((20, 21, 22)) + 0.05
    m = rng.integers(5, size=J.shape) % 4 == 0
    P = J.copy()
    P[m] = 0.05 - rng.random()
    R = dt.regularise(P, 0.05)
    assert np.array_equal(R[~m], J[~m])
    assert np.all(R[m] == 0.05)


def test_extension_jacobian_matches(golden):
    from disptools_b200 import _disptools
    g = golden["jacobian"]
    out = np.zeros((10, 10, 10))
    _disptools.jacobian((1.0, 1.0, 1.0), g["sin10_field"], out)
    np.testing.assert_array_equal(out, g["sin10_J"])
