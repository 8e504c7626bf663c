"""disptools_b200 — B200-native (sm_100a) displacement-field generator.

Drop-in for the hot path of disptools v0.4.1: the finite-difference Jacobian
determinant, the masked Jacobian-error cost and its gradient, the
Armijo-controlled gradient method and the greedy method.  All compute runs in
hand-written CUDA kernels in ``libdisptools_b200.so``; there is no CPU path.

* ``disptools_b200._disptools`` — NumPy extension with the reference
  ``_disptools`` method table;
* ``disptools_b200.api`` — NumPy functions with statistics and batching;
* ``disptools_b200.torch_ops`` — device-tensor entry points and the
  differentiable ``jacobian`` (torch is only needed there).

The CUDA library is loaded on first use of any of the names below (or on
import of ``_native``, ``api``, ``torch_ops`` …), and that fails loudly when
the library is missing.  Modules that compute nothing on the device, such as
``disptools_b200.synthetic`` and ``disptools_b200.sharding``, import without
loading it.
"""
from __future__ import annotations

_NATIVE = ("DisptoolsError", "lib")
_API = ("jacobian", "kernel_launch_count", "kernel_profile", "regularise", "release_device_memory",
        "set_autotune", "set_default_precision", "set_profiling", "set_verbose", "solve",
        "solve_batched", "tile_config")

__all__ = list(_NATIVE + _API)
__version__ = "0.1.0"


def __getattr__(name):
    if name in _NATIVE:
        from . import _native
        return getattr(_native, name)
    if name in _API:
        from . import api
        return getattr(api, name)
    raise AttributeError(f"module 'disptools_b200' has no attribute {name!r}")
