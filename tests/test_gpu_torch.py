"""The differentiable Jacobian: adjoint kernel against FP64 central finite
differences and against the reference's analytic gradient (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _affected(shape, q):
    """Voxels whose Jacobian reads voxel q (the radius-2 cross)."""
    out = []
    for a in range(3):
        for t in range(-2, 3):
            p = list(q)
            p[a] += t
            if all(0 <= p[i] < shape[i] for i in range(3)) and (a == 0 or t != 0):
                out.append(tuple(p))
    return out


def fd_check(field64, w, grad, probes, spacing=(1.0, 1.0, 1.0), h=1e-6, order=4):
    """Central differences of L = sum w J(u) at `probes` (component, z, y, x),
    differenced only over the voxels each probe affects."""
    import torch
    from disptools_b200 import torch_ops
    fd = []
    for c, z, y, x in probes:
        f = field64.clone()
        f[c, z, y, x] += h
        Jp = torch_ops.jacobian_raw(f, spacing, order)
        f[c, z, y, x] -= 2 * h
        Jm = torch_ops.jacobian_raw(f, spacing, order)
        idx = _affected(field64.shape[1:], (z, y, x))
        zi, yi, xi = (torch.tensor(v, device=f.device) for v in zip(*idx))
        fd.append(float(torch.sum(w[zi, yi, xi] * (Jp[zi, yi, xi] - Jm[zi, yi, xi]))) / (2 * h))
    got = np.array([float(grad[c, z, y, x]) for c, z, y, x in probes])
    return got, np.array(fd)


@pytest.mark.parametrize("shape", [(14, 12, 10), (13, 11, 19)])
def test_adjoint_fp64_vs_finite_differences(shape):
    """The second shape has odd extents and a deep interior along x, where
    the gather uses its constant weights."""
    import torch
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    f = torch.from_numpy(smooth_field(shape, sigma=2.0, max_disp=0.8, seed=1)).cuda()
    f.requires_grad_(True)
    rng = np.random.default_rng(2)
    w = torch.from_numpy(rng.standard_normal(shape)).cuda()
    sp = (0.9, 1.1, 1.3)
    J = torch_ops.jacobian(f, sp)
    (J * w).sum().backward()
    probes = [(int(c), int(z), int(y), int(x)) for c, z, y, x in
              zip(rng.integers(0, 3, 300), rng.integers(0, shape[0], 300), rng.integers(0, shape[1], 300),
                  rng.integers(0, shape[2], 300))]
    got, fd = fd_check(f.detach(), w, f.grad, probes, sp)
    np.testing.assert_allclose(got, fd, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("shape", [(21, 40, 68), (96, 112, 100)])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_adjoint_tma_and_plain_paths_agree(dtype, shape):
    """The TMA passes (aligned field: weight pass on the TMA stencil kernel,
    TMA gather) and the plain-load passes (a field 8 bytes off a 16-byte
    boundary) give the same gradient on every voxel: several tiles per axis,
    tiles on every face (the gather's x-face and general paths) and a deep
    interior (its fourth-order path); bit for bit in FP64."""
    import torch
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    tdt = getattr(torch, dtype)
    f = torch.from_numpy(smooth_field(shape, sigma=3.0, max_disp=1.5, seed=4)).to(tdt).cuda()
    rng = np.random.default_rng(5)
    w = torch.from_numpy(rng.standard_normal(shape)).to(tdt).cuda()
    sp = (0.9, 1.2, 1.05)
    g_tma = torch_ops.jacobian_adjoint_raw(f, w, sp)
    k = 8 // f.element_size()  # elements in 8 bytes
    buf = torch.zeros(f.numel() + k, dtype=tdt, device="cuda")
    buf[k:] = f.reshape(-1)
    off = buf[k:].view(f.shape)
    assert off.data_ptr() % 16 == 8
    g_plain = torch_ops.jacobian_adjoint_raw(off, w, sp)
    if dtype == "float64":
        torch.testing.assert_close(g_tma, g_plain, rtol=0, atol=0)
    else:
        torch.testing.assert_close(g_tma, g_plain, rtol=1e-5, atol=1e-5)


def test_adjoint_matches_reference_gradient(oracle_pd2):
    """With second-order differences the cost gradient of the reference
    (src/displacement_field_gradient.c:26-145) is the adjoint applied to
    2 e' (e' the regularised error), on voxels away from the boundary."""
    import torch
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    shape = (16, 15, 14)
    f = smooth_field(shape, sigma=2.0, max_disp=1.5, seed=3)
    rng = np.random.default_rng(4)
    Jt = 1.0 + 0.1 * rng.standard_normal(shape)
    mask = rng.random(shape) < 0.5
    sp = (1.0, 1.2, 0.8)
    delta, zeta = 0.9, 10.0  # a delta above some J values exercises the regulariser
    J2 = oracle_pd2.jacobian(f, sp)
    _, _, v = oracle_pd2.compute_error(Jt, J2, mask, 0.2)
    g_ref, _ = oracle_pd2.gradient(f, J2, v, delta, zeta, sp)
    ep = v + np.where(J2 < delta, zeta * (J2 - delta), 0.0)
    g = torch_ops.jacobian_adjoint_raw(torch.from_numpy(f).cuda(), torch.from_numpy(2 * ep).cuda(),
                                       sp, order=2).cpu().numpy()
    inner = (slice(None),) + (slice(3, -3),) * 3
    np.testing.assert_allclose(g[inner], g_ref[inner], rtol=1e-10, atol=1e-12)


def test_batched_fp32_autograd_config3():
    """4 fields of 192x224x192 (smooth noise, sigma 6, max |u| = 3): FP32
    forward and backward; the backward checked on 1000 random voxels against
    FP64 central differences (h = 1e-6)."""
    import torch
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    shape = (192, 224, 192)
    fields = np.stack([smooth_field(shape, 6.0, 3.0, seed=s) for s in range(4)])
    f32 = torch.from_numpy(fields).float().cuda().requires_grad_(True)
    rng = np.random.default_rng(9)
    w = torch.from_numpy(rng.standard_normal((4,) + shape)).cuda()
    J = torch_ops.jacobian(f32)
    assert J.shape == (4,) + shape
    (J * w.float()).sum().backward()
    g = f32.grad
    errs = []
    for b in range(4):
        f64 = torch.from_numpy(fields[b]).cuda()
        probes = [(int(c), int(z), int(y), int(x)) for c, z, y, x in
                  zip(rng.integers(0, 3, 250), rng.integers(0, shape[0], 250),
                      rng.integers(0, shape[1], 250), rng.integers(0, shape[2], 250))]
        got, fd = fd_check(f64, w[b], g[b], probes)
        scale = np.maximum(np.abs(fd), 1.0)
        errs.append(np.max(np.abs(got - fd) / scale))
    assert max(errs) <= 1e-4, errs


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("shape", [(3, 3, 4), (5, 9, 12), (7, 17, 36), (40, 40, 96), (37, 21, 100),
                                   (30, 53, 132)])
def test_fused_adjoint_equals_two_pass(monkeypatch, dtype, shape):
    """The fused adjoint kernel (one launch, weights on chip,
    DISPTOOLS_B200_ADJOINT=fused) against the weight pass + gather: bit for bit in
    FP64, to float rounding in FP32.  The shapes give partial tiles on every
    axis, volumes of 3 voxels, and (40 x 40 x 96) tiles whose every voxel is
    four cells from the faces (the constant-weight path)."""
    import torch

    import disptools_b200 as dt
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    t = getattr(torch, dtype)
    f = torch.from_numpy(smooth_field(shape, sigma=2.0, max_disp=0.8, seed=3)).to(t).cuda()
    w = torch.from_numpy(np.random.default_rng(4).standard_normal(shape)).to(t).cuda()
    sp = (0.9, 1.1, 1.3)
    monkeypatch.setenv("DISPTOOLS_B200_ADJOINT", "fused")
    n0 = dt.kernel_launch_count()
    fused = torch_ops.jacobian_adjoint_raw(f, w, sp)
    torch.cuda.synchronize()
    assert dt.kernel_launch_count() - n0 == 1  # one kernel: the fused path ran
    monkeypatch.delenv("DISPTOOLS_B200_ADJOINT")
    n0 = dt.kernel_launch_count()
    two = torch_ops.jacobian_adjoint_raw(f, w, sp)
    torch.cuda.synchronize()
    assert dt.kernel_launch_count() - n0 == 2
    a, b = fused.cpu().numpy(), two.cpu().numpy()
    if dtype == "float64":
        np.testing.assert_array_equal(a, b)
    else:
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(b).max())


@pytest.mark.parametrize("shape", [(3, 3, 4), (7, 17, 36), (21, 40, 68), (40, 40, 96), (30, 53, 132)])
def test_autograd_cofactor_path_matches_weight_path(monkeypatch, shape):
    """The FP32 autograd forward that keeps C = cof * ih and the one-gather
    backward (the default for TMA-friendly layouts) against the weight pass +
    gather (DISPTOOLS_B200_AUTOGRAD=weights): the same map bit for bit, the
    same gradient to float rounding (grad_J * (cof * ih) against
    (grad_J * cof) * ih); single and batched fields."""
    import torch
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field
    fields = np.stack([smooth_field(shape, sigma=2.0, max_disp=0.8, seed=s) for s in (3, 4)])
    w = torch.from_numpy(np.random.default_rng(5).standard_normal((2,) + shape)).float().cuda()
    sp = (0.9, 1.1, 1.3)

    def run(batched):
        f = torch.from_numpy(fields).float().cuda().requires_grad_(True)
        if batched:
            J = torch_ops.jacobian(f, sp)
            (J * w).sum().backward()
        else:
            J = torch.stack([torch_ops.jacobian(f[b], sp) for b in range(2)])
            (J * w).sum().backward()
        return J.detach(), f.grad

    assert torch_ops.cof_supported(torch.zeros((3,) + shape, device="cuda"))
    for batched in (False, True):
        Jc, gc = run(batched)
        monkeypatch.setenv("DISPTOOLS_B200_AUTOGRAD", "weights")
        Jw, gw = run(batched)
        monkeypatch.delenv("DISPTOOLS_B200_AUTOGRAD")
        torch.testing.assert_close(Jc, Jw, rtol=0, atol=0)
        scale = gw.abs().max().item()
        torch.testing.assert_close(gc, gw, rtol=1e-5, atol=1e-6 * scale)


def test_autograd_cofactor_path_unsupported_layouts_fall_back():
    """Widths that are not a multiple of four float32 elements and float64
    fields take the weight pass + gather."""
    import torch
    from disptools_b200 import torch_ops
    assert not torch_ops.cof_supported(torch.zeros((3, 8, 8, 9), device="cuda"))
    assert not torch_ops.cof_supported(torch.zeros((3, 8, 8, 8), dtype=torch.float64, device="cuda"))
    f = torch.rand((3, 8, 8, 9), device="cuda", requires_grad=True)
    torch_ops.jacobian(f).sum().backward()
    assert f.grad is not None and torch.isfinite(f.grad).all()


def test_cof_entry_points_reject_unsupported_layouts():
    """The C entry points of the cofactor path refuse layouts their tensor
    maps cannot cover (rows not a multiple of 16 bytes, misaligned bases)
    with DTB_ERR_ARGUMENT and the error state set, and do no device work."""
    import torch
    from disptools_b200 import _native as N
    f = torch.zeros((3, 8, 8, 9), device="cuda")
    J = torch.zeros((8, 8, 9), device="cuda")
    C = torch.zeros((9, 8, 8, 9), device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = N.lib.dtb_jacobian_cof_device(N.PRECISION_MIXED, 9, 8, 8, 1.0, 1.0, 1.0, f.data_ptr(), J.data_ptr(),
                                       C.data_ptr(), s)
    assert rc == -1 and N.lib.disptools_has_error()
    buf = torch.zeros(9 * 8 * 8 * 8 + 1, device="cuda")
    C8 = buf[1:]  # 4 bytes off the allocation's alignment
    gJ = torch.zeros((8, 8, 8), device="cuda")
    g = torch.zeros((3, 8, 8, 8), device="cuda")
    rc = N.lib.dtb_jacobian_adjoint_cof_device(N.PRECISION_MIXED, 8, 8, 8, 1.0, 1.0, 1.0, C8.data_ptr(),
                                               gJ.data_ptr(), g.data_ptr(), s)
    assert rc == -1 and N.lib.disptools_has_error()
    N.lib.disptools_clear_error()
