"""dtb_jacobian_device_noalloc: the Jacobian entry point for callers that
cannot let the library allocate device memory — hosts whose memory budget is
fixed at start-up, processes whose device memory another allocator has
reserved, runtimes that hand the library pointers into memory they manage.
Its results must equal those of dtb_jacobian_device and of the FP64 oracle,
call after call, although every call reuses the same fixed scratch array.

This file is collected last so that a failure here does not stop the rest of
the suite early."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jacobians(torch, N, field, spacing, order):
    nz, ny, nx = field.shape[1:]
    prec = N.PRECISION_FP64 if field.dtype == torch.float64 else N.PRECISION_MIXED
    ref = torch.empty((nz, ny, nx), dtype=field.dtype, device=field.device)
    new = torch.full((nz, ny, nx), float("nan"), dtype=field.dtype, device=field.device)
    stream = torch.cuda.current_stream().cuda_stream
    N.check(N.lib.dtb_jacobian_device(prec, order, nx, ny, nz, *spacing, field.data_ptr(),
                                      ref.data_ptr(), stream))
    N.check(N.lib.dtb_jacobian_device_noalloc(prec, order, nx, ny, nz, *spacing, field.data_ptr(),
                                              new.data_ptr(), stream))
    torch.cuda.synchronize()
    return ref.cpu().numpy(), new.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(oracle, oracle_pd2):
    import torch
    from disptools_b200 import _native as N
    rng = np.random.default_rng(12)
    # consecutive calls with different shapes, precisions and orders: the
    # shared scratch must not carry anything over from the previous call
    cases = [((21, 34, 45), torch.float64, (0.9, 1.2, 1.05), 4),
             ((40, 17, 70), torch.float32, (1.0, 1.0, 1.0), 4),
             ((3, 9, 5), torch.float64, (2.0, 3.0, 4.0), 2),
             ((21, 34, 45), torch.float64, (0.9, 1.2, 1.05), 4)]
    for shape, dtype, spacing, order in cases:
        f64 = rng.normal(scale=0.2, size=(3,) + shape)
        f = torch.from_numpy(f64).to(dtype).cuda()
        ref, new = _jacobians(torch, N, f, spacing, order)
        # same kernel and arithmetic: identical up to the FP64 tolerance of the suite
        rel = np.max(np.abs(new - ref) / np.maximum(np.abs(ref), 1.0))
        assert rel <= 1e-12, (shape, dtype, rel)
        # and against the oracle on the field the device saw: 1e-12 relative
        # in FP64, the suite's FP32 bound (1e-4) in FP32
        o = (oracle if order == 4 else oracle_pd2).jacobian(f.double().cpu().numpy(), spacing)
        tol = 1e-12 if dtype == torch.float64 else 1e-4
        rel_o = np.max(np.abs(new - o) / np.maximum(np.abs(o), 1.0))
        assert rel_o <= tol, (shape, dtype, rel_o)


def test_noalloc_rejects_volumes_beyond_its_scratch():
    import torch
    from disptools_b200 import _native as N
    # 1024 x 1024 x 160 voxels need 32 x 128 x 5 = 20480 tiles of 32 x 8 x 32,
    # more than the 16384 the fixed scratch holds: rejected before any GPU work.
    dummy = torch.zeros(1, device="cuda")
    rc = N.lib.dtb_jacobian_device_noalloc(N.PRECISION_MIXED, 4, 1024, 1024, 160, 1.0, 1.0, 1.0,
                                           dummy.data_ptr(), dummy.data_ptr(), None)
    assert rc == N.ERR_ARGUMENT
    assert b"too large" in N.lib.disptools_get_error().contents.message
    N.lib.disptools_clear_error()
