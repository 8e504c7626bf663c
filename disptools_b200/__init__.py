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
"""
from ._native import DisptoolsError, lib  # noqa: F401  (loads the CUDA library)
from .api import (jacobian, kernel_launch_count, kernel_profile, regularise,  # noqa: F401
                  release_device_memory, set_autotune, set_default_precision, set_profiling,
                  set_verbose, solve, solve_batched, tile_config)

__version__ = "0.1.0"
