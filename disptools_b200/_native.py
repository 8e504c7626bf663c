"""ctypes bindings of ``libdisptools_b200.so`` (the C ABI in
``include/disptools_b200.h``).

Importing this module loads the CUDA library.  There is no fallback: if the
library is missing the import fails with instructions to build it.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libdisptools_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build the CUDA library with "
        "`python disptools_b200/build.py` (nvcc with sm_100a support is required)")

lib = C.CDLL(LIB_PATH)

PRECISION_MIXED = 0
PRECISION_FP64 = 1
ALGORITHM_GRADIENT = 0
ALGORITHM_GREEDY = 1
ALGORITHM_MATCHING = 2

OK = 0
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_ALLOC = -3
ERR_DEVICE = -4
ERR_IO = -5

STOP_REASONS = {
    0: "it_max",
    1: "error exploded",
    2: "eta < iota",
    3: "improvement < theta",
    4: "voxel error exploded",
    5: "tolerance reached",
}


class ErrorState(C.Structure):
    _fields_ = [
        ("error", C.c_bool),
        ("line", C.c_int),
        ("file", C.c_char * 512),
        ("function", C.c_char * 512),
        ("message", C.c_char * 1024),
        ("trace", C.c_char * 4096),
    ]


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("epsilon", "tolerance", "eta", "eta_max", "alpha", "beta", "gamma", "delta",
                 "zeta", "theta", "iota")] + [("strict", C.c_int), ("it_max", C.c_longlong)]


class SolveStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_longlong),
        ("trials", C.c_longlong),
        ("gradients", C.c_longlong),
        ("reason", C.c_int),
        ("precision", C.c_int),
        ("error", C.c_double),
        ("max_error", C.c_double),
        ("cand_error", C.c_double),
        ("cand_max_error", C.c_double),
        ("eta", C.c_double),
        ("device_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["reason"] = STOP_REASONS.get(self.reason, str(self.reason))
        d["precision"] = "fp64" if self.precision == PRECISION_FP64 else "mixed"
        return d


class Volume(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("J", C.c_void_p), ("mask", C.c_void_p), ("field", C.c_void_p)]


DeviceVolume = Volume  # same layout: dtb_device_volume

_D, _SZ, _P, _I = C.c_double, C.c_size_t, C.c_void_p, C.c_int

lib.disptools_get_error.restype = C.POINTER(ErrorState)
lib.disptools_has_error.restype = C.c_bool
lib.get_float_type_size.restype = _I
lib.set_device.argtypes = [_I]
lib.set_device.restype = C.c_bool
_REF_SOLVER = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P] + [_D] * 11 + [C.c_bool, _SZ, _P]
lib.generate_displacement_gradient_cuda.argtypes = _REF_SOLVER
lib.generate_displacement_gradient_cuda.restype = None
lib.generate_displacement_greedy_cuda.argtypes = _REF_SOLVER
lib.generate_displacement_greedy_cuda.restype = None
lib.jacobian_dynamic.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P]
lib.jacobian_dynamic.restype = None
lib.regularise.argtypes = [_SZ, _SZ, _SZ, _P, _D]
lib.regularise.restype = None
lib.dtb_set_default_precision.argtypes = [_I]
lib.dtb_set_default_precision.restype = _I
lib.dtb_get_default_precision.restype = _I
lib.dtb_generate_displacement.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P,
                                          C.POINTER(Params), _P, C.POINTER(SolveStats)]
lib.dtb_generate_displacement.restype = _I
lib.dtb_generate_displacement_batched.argtypes = [_I, _I, _I, C.POINTER(Volume), C.POINTER(Params),
                                                  C.POINTER(SolveStats)]
lib.dtb_generate_displacement_batched.restype = _I
lib.dtb_generate_displacement_batched_device.argtypes = [_I, _I, _I, C.POINTER(Volume),
                                                         C.POINTER(Params), C.POINTER(SolveStats), _P]
lib.dtb_generate_displacement_batched_device.restype = _I
lib.dtb_jacobian_device.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P]
lib.dtb_jacobian_device.restype = _I
lib.dtb_jacobian_device_noalloc.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P]
lib.dtb_jacobian_device_noalloc.restype = _I
lib.dtb_jacobian_adjoint_device.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _P]
lib.dtb_jacobian_adjoint_device.restype = _I
lib.dtb_jacobian_cof_device.argtypes = [_I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _P]
lib.dtb_jacobian_cof_device.restype = _I
lib.dtb_jacobian_adjoint_cof_device.argtypes = [_I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _P]
lib.dtb_jacobian_adjoint_cof_device.restype = _I
lib.dtb_kernel_launch_count.restype = C.c_ulonglong
lib.dtb_release_device_memory.argtypes = []
lib.dtb_release_device_memory.restype = _I
lib.dtb_smooth_device.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _P]
lib.dtb_smooth_device.restype = _I
lib.dtb_smooth_recursive_device.argtypes = [_I, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _P]
lib.dtb_smooth_recursive_device.restype = _I
lib.dtb_resample_device.argtypes = [_I, _I, _I, _SZ, _SZ, _SZ, _SZ, _SZ, _SZ, _P, _P, _P]
lib.dtb_resample_device.restype = _I
_SZP, _DP = C.POINTER(C.c_size_t), C.POINTER(C.c_double)
lib.dtb_write_rvf.argtypes = [C.c_char_p, _SZ, _SZ, _SZ, _D, _D, _D, _P]
lib.dtb_write_rvf.restype = _I
lib.dtb_read_rvf_header.argtypes = [C.c_char_p, _SZP, _SZP, _SZP, _DP, _DP, _DP]
lib.dtb_read_rvf_header.restype = _I
lib.dtb_read_rvf.argtypes = [C.c_char_p, _P, _SZ]
lib.dtb_read_rvf.restype = _I
lib.dtb_write_vtk.argtypes = [C.c_char_p, _I, _SZ, _SZ, _SZ, _D, _D, _D, _P]
lib.dtb_write_vtk.restype = _I
lib.dtb_read_vtk_header.argtypes = [C.c_char_p, C.POINTER(C.c_int), _SZP, _SZP, _SZP, _DP, _DP, _DP]
lib.dtb_read_vtk_header.restype = _I
lib.dtb_read_vtk.argtypes = [C.c_char_p, _P, _SZ]
lib.dtb_read_vtk.restype = _I
lib.dtb_volume_change_device.argtypes = [_I, _SZ, _D, _P, _P, _P]
lib.dtb_volume_change_device.restype = _I
lib.dtb_log_jacobian_accumulate_device.argtypes = [_I, _I, _SZ, _D, _P, _P, _P]
lib.dtb_log_jacobian_accumulate_device.restype = _I
lib.dtb_exp_mean_device.argtypes = [_I, _SZ, _D, _P, _P, _P]
lib.dtb_exp_mean_device.restype = _I
lib.volume_matching_3d.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P] + [_D] * 11 + [C.c_bool, _SZ, _P]
lib.volume_matching_3d.restype = None
lib.dtb_volume_matching.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P, C.POINTER(Params), _P,
                                    C.POINTER(SolveStats)]
lib.dtb_volume_matching.restype = _I
lib.dtb_volume_matching_device.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, C.POINTER(Params), _P,
                                           C.POINTER(SolveStats), _P]
lib.dtb_volume_matching_device.restype = _I
lib.dtb_set_device_memory_limit.argtypes = [_SZ]
lib.dtb_set_device_memory_limit.restype = _I
lib.dtb_test_drop_tma_load.argtypes = [C.c_longlong, _I, C.c_uint]
lib.dtb_test_drop_tma_load.restype = _I
lib.dtb_set_verbose.argtypes = [_I]
lib.dtb_set_verbose.restype = _I
lib.dtb_set_autotune.argtypes = [_I]
lib.dtb_set_autotune.restype = _I
lib.dtb_get_tile_config.argtypes = [C.POINTER(C.c_int)]
lib.dtb_get_tile_config.restype = _I
lib.dtb_get_trial_kernel.argtypes = []
lib.dtb_get_trial_kernel.restype = _I


class KernelProfile(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("total_ms", C.c_double)]


lib.dtb_set_profiling.argtypes = [_I]
lib.dtb_set_profiling.restype = _I
lib.dtb_get_profile.argtypes = [C.POINTER(KernelProfile), _I]
lib.dtb_get_profile.restype = _I

# Every symbol declared in include/disptools_b200.h.
EXPORTED = [
    "disptools_get_error", "disptools_has_error", "disptools_clear_error", "get_float_type_size",
    "set_device", "generate_displacement_gradient_cuda", "generate_displacement_greedy_cuda",
    "jacobian_dynamic", "regularise", "dtb_set_default_precision", "dtb_get_default_precision",
    "dtb_generate_displacement", "dtb_generate_displacement_batched",
    "dtb_generate_displacement_batched_device", "dtb_jacobian_device",
    "dtb_jacobian_adjoint_device", "dtb_jacobian_cof_device", "dtb_jacobian_adjoint_cof_device",
    "dtb_kernel_launch_count", "dtb_set_profiling",
    "dtb_get_profile", "dtb_jacobian_device_noalloc", "dtb_release_device_memory",
    "dtb_set_autotune", "dtb_get_tile_config", "dtb_get_trial_kernel", "dtb_smooth_device",
    "dtb_smooth_recursive_device", "dtb_resample_device",
    "dtb_write_rvf", "dtb_read_rvf_header", "dtb_read_rvf", "dtb_write_vtk", "dtb_read_vtk_header",
    "dtb_read_vtk", "dtb_volume_change_device", "dtb_log_jacobian_accumulate_device",
    "dtb_exp_mean_device", "volume_matching_3d", "dtb_volume_matching", "dtb_volume_matching_device",
    "dtb_set_verbose",
    "dtb_set_device_memory_limit", "dtb_test_drop_tma_load",
]


class DisptoolsError(RuntimeError):
    pass


def last_error() -> str:
    e = lib.disptools_get_error().contents
    return (f"{e.function.decode()} ({e.file.decode()}:{e.line}): {e.message.decode()}"
            if e.error else "")


def check(rc: int) -> None:
    if rc != OK or lib.disptools_has_error():
        msg = last_error() or f"error code {rc}"
        if rc == ERR_ARGUMENT:
            raise ValueError(msg)
        if rc == ERR_IO:
            raise OSError(msg)
        raise DisptoolsError(msg)


def precision_code(precision) -> int:
    if precision in (PRECISION_MIXED, "mixed", "fp32", "float32"):
        return PRECISION_MIXED
    if precision in (PRECISION_FP64, "fp64", "float64", "double"):
        return PRECISION_FP64
    raise ValueError(f"unknown precision {precision!r}")


def algorithm_code(algorithm) -> int:
    if algorithm in (ALGORITHM_GRADIENT, "gradient"):
        return ALGORITHM_GRADIENT
    if algorithm in (ALGORITHM_GREEDY, "greedy"):
        return ALGORITHM_GREEDY
    if algorithm in (ALGORITHM_MATCHING, "matching"):
        return ALGORITHM_MATCHING
    raise ValueError(f"Invalid algorithm '{algorithm}'.")
