"""ctypes access to the CPU oracle (test infrastructure only).

Loads the restatement built from ``oracle/dt_oracle.c`` (``liboracle64.so``,
``liboracle64_pd2.so``) and, when present, the reference C library compiled
from its own sources into ``oracle/_ref/`` by ``oracle/Makefile``.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The disptools_b200 product never does.

Array conventions are those of the reference C ABI (src/headers/disptools.h):
fields are C-contiguous ``[3, nz, ny, nx]`` float64, scalar maps
``[nz, ny, nx]``, masks ``bool``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

STOP_REASONS = {
    0: "it_max",
    1: "error exploded",
    2: "eta < iota",
    3: "improvement < theta",
    4: "voxel error exploded",
    5: "tolerance reached",
    6: "allocation failed",
}


class _Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_long),
        ("trials", C.c_long),
        ("gradients", C.c_long),
        ("reason", C.c_int),
        ("error", C.c_double),
        ("max_error", C.c_double),
        ("cand_error", C.c_double),
        ("cand_max_error", C.c_double),
        ("eta", C.c_double),
    ]


@dataclass
class SolveStats:
    iterations: int
    trials: int
    gradients: int
    reason: str
    error: float
    max_error: float
    cand_error: float
    cand_max_error: float
    eta: float


def reference_dir() -> str:
    """Where the reference checkout lies: $DISPTOOLS_REFERENCE, else the
    default location of this build environment.  The only place that names
    it; the GPU-side runs use the libraries already built into _ref/."""
    return os.environ.get("DISPTOOLS_REFERENCE", "/root/reference")


def build(ref: bool | None = None) -> None:
    """Build the oracle (and the reference libraries when the reference
    sources are reachable)."""
    ref_src = reference_dir()
    targets = ["oracle"]
    if ref is None:
        ref = os.path.isdir(os.path.join(ref_src, "src"))
    if ref:
        targets += ["ref", "refext"]
    subprocess.check_call(["make", "-s", "-C", HERE, f"REF={ref_src}", *targets])


_D = C.c_double
_SZ = C.c_size_t
_P = C.c_void_p
_SOLVER_ARGS = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P,
                _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, C.c_bool, _SZ, _P]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _f64(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class Oracle:
    """The FP64 restatement (``order_pd`` 4 by default, or 2)."""

    def __init__(self, order_pd: int = 4):
        name = "liboracle64.so" if order_pd == 4 else "liboracle64_pd2.so"
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build(ref=False)
        lib = C.CDLL(path)
        lib.oracle_jacobian.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P]
        lib.oracle_jacobian.restype = None
        lib.oracle_regularise.argtypes = [_SZ, _SZ, _SZ, _P, _D]
        lib.oracle_compute_error.argtypes = [_SZ, _P, _P, _P, _D, _P, _P]
        lib.oracle_compute_error.restype = _D
        lib.oracle_gradient.argtypes = [_SZ, _SZ, _SZ, _D, _D, _D, _P, _P, _P, _D, _D, _P, _P]
        for fn in (lib.oracle_generate_gradient, lib.oracle_generate_greedy):
            fn.argtypes = _SOLVER_ARGS + [C.POINTER(_Stats)]
            fn.restype = C.c_int
        self.lib = lib
        self.order_pd = lib.oracle_order_pd()

    # -- a1/a2 ---------------------------------------------------------
    def jacobian(self, field: np.ndarray, spacing=(1.0, 1.0, 1.0)) -> np.ndarray:
        field = _f64(field)
        _, nz, ny, nx = field.shape
        J = np.zeros((nz, ny, nx), np.float64)
        self.lib.oracle_jacobian(nx, ny, nz, *map(float, spacing), _ptr(field), _ptr(J))
        return J

    def regularise(self, J: np.ndarray, epsilon: float) -> np.ndarray:
        J = _f64(J).copy()
        nz, ny, nx = J.shape
        self.lib.oracle_regularise(nx, ny, nz, _ptr(J), float(epsilon))
        return J

    # -- a3 ------------------------------------------------------------
    def compute_error(self, Jt, Jf, mask, tolerance):
        Jt = _f64(Jt)
        Jf = _f64(Jf, Jt.shape)
        mask = np.ascontiguousarray(mask, dtype=np.bool_)
        v = np.zeros_like(Jt)
        mx = np.zeros(1, np.float64)
        tot = self.lib.oracle_compute_error(Jt.size, _ptr(Jt), _ptr(Jf), _ptr(mask),
                                            float(tolerance), _ptr(v), _ptr(mx))
        return tot, float(mx[0]), v

    # -- a4 ------------------------------------------------------------
    def gradient(self, field, Jf, v, delta, zeta, spacing=(1.0, 1.0, 1.0)):
        field = _f64(field)
        _, nz, ny, nx = field.shape
        Jf = _f64(Jf, (nz, ny, nx))
        v = _f64(v, (nz, ny, nx))
        g = np.zeros_like(field)
        gn2 = np.zeros(1, np.float64)
        self.lib.oracle_gradient(nx, ny, nz, *map(float, spacing), _ptr(field), _ptr(Jf),
                                 _ptr(v), float(delta), float(zeta), _ptr(g), _ptr(gn2))
        return g, float(gn2[0])

    # -- a6/a7 ---------------------------------------------------------
    def solve(self, algorithm, Jt, mask, field=None, spacing=(1.0, 1.0, 1.0), **params):
        Jt = _f64(Jt)
        nz, ny, nx = Jt.shape
        mask = np.ascontiguousarray(mask, dtype=np.bool_)
        out = np.zeros((3, nz, ny, nx)) if field is None else _f64(field, (3, nz, ny, nx)).copy()
        p = solver_params(**params)
        st = _Stats()
        fn = {"gradient": self.lib.oracle_generate_gradient,
              "greedy": self.lib.oracle_generate_greedy}[algorithm]
        rc = fn(nx, ny, nz, *map(float, spacing), _ptr(Jt), _ptr(mask), *p, _ptr(out), C.byref(st))
        if rc != 0:
            raise MemoryError("oracle allocation failed")
        return out, SolveStats(st.iterations, st.trials, st.gradients,
                               STOP_REASONS.get(st.reason, str(st.reason)), st.error,
                               st.max_error, st.cand_error, st.cand_max_error, st.eta)


DEFAULTS = dict(epsilon=9.99e-4, tolerance=0.2, eta=0.1, eta_max=0.4, alpha=1.2, beta=0.5,
                gamma=0.1, delta=1e-3, zeta=10.0, theta=1e-6, iota=1e-9, strict=False,
                it_max=50000)
_ORDER = ["epsilon", "tolerance", "eta", "eta_max", "alpha", "beta", "gamma", "delta",
          "zeta", "theta", "iota", "strict", "it_max"]


def solver_params(**params):
    """The 13 scalar solver parameters in C-ABI order, defaults from the
    reference Python wrapper (disptools/displacements.py:238-260)."""
    unknown = set(params) - set(DEFAULTS)
    if unknown:
        raise TypeError(f"unknown solver parameters {sorted(unknown)}")
    p = {**DEFAULTS, **params}
    out = []
    for k in _ORDER:
        if k == "strict":
            out.append(bool(p[k]))
        elif k == "it_max":
            out.append(int(p[k]))
        else:
            out.append(float(p[k]))
    return out


def reference_extension():
    """The reference's own ``_disptools`` extension module compiled against
    the drop-in library (``make refext``), or None when it was not built."""
    import glob
    import importlib.machinery
    import importlib.util
    paths = glob.glob(os.path.join(REF_DIR, "refext", "_disptools*.so"))
    if not paths:
        return None
    loader = importlib.machinery.ExtensionFileLoader("_disptools", paths[0])
    spec = importlib.util.spec_from_file_location("_disptools", paths[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


class Reference:
    """The reference C library compiled from its own sources (FP64 or FP32
    FLOATING; ORDER_PD 4, or 2 for ``libdisptools_ref64_pd2``;
    ``libdisptools_ref64_match`` holds the matching solver)."""

    def __init__(self, flavour: str = "ref64"):
        path = os.path.join(REF_DIR, f"libdisptools_{flavour}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        self.dtype = np.float64 if lib.get_float_type_size() == 64 else np.float32
        R = C.c_double if self.dtype == np.float64 else C.c_float
        if hasattr(lib, "jacobian_dynamic"):
            lib.jacobian_dynamic.argtypes = [_SZ, _SZ, _SZ, R, R, R, _P, _P]
            lib.regularise.argtypes = [_SZ, _SZ, _SZ, _P, R]
        args = [_SZ, _SZ, _SZ, R, R, R, _P, _P] + [R] * 11 + [C.c_bool, _SZ, _P]
        if hasattr(lib, "generate_displacement_gradient"):
            lib.generate_displacement_gradient.argtypes = args
            lib.generate_displacement_greedy.argtypes = args
        if hasattr(lib, "volume_matching_3d"):
            lib.volume_matching_3d.argtypes = args
        lib.disptools_has_error.restype = C.c_bool
        self.lib = lib

    @staticmethod
    def available(flavour: str = "ref64") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libdisptools_{flavour}.so"))

    def jacobian(self, field, spacing=(1.0, 1.0, 1.0)):
        field = np.ascontiguousarray(field, dtype=self.dtype)
        _, nz, ny, nx = field.shape
        J = np.zeros((nz, ny, nx), self.dtype)
        self.lib.jacobian_dynamic(nx, ny, nz, *map(float, spacing), _ptr(field), _ptr(J))
        return J

    def regularise(self, J, epsilon):
        J = np.ascontiguousarray(J, dtype=self.dtype).copy()
        nz, ny, nx = J.shape
        self.lib.regularise(nx, ny, nz, _ptr(J), float(epsilon))
        return J

    def solve_logged(self, algorithm, Jt, mask, field=None, spacing=(1.0, 1.0, 1.0), **params):
        """``solve`` with the library's standard output captured at the file
        descriptor (the verbose build, ``ref64_verbose``, prints one
        ``Iteration`` line per pass of its loop, src/displacement_field_gradient.c:378,
        src/displacement_field_greedy.c:184).  Returns the field, the output
        lines and the iterations completed: the largest number printed on an
        ``Iteration`` line (the loop counter; iteration 0 is the initial
        field, src/displacement_field_gradient.c:272, and the greedy method
        prints a rejected step again under the same number,
        src/displacement_field_greedy.c:209-212)."""
        import sys
        import tempfile
        libc = C.CDLL(None)
        sys.stdout.flush()
        saved = os.dup(1)
        with tempfile.TemporaryFile(mode="w+b") as tmp:
            os.dup2(tmp.fileno(), 1)
            try:
                out = self.solve(algorithm, Jt, mask, field, spacing, **params)
            finally:
                libc.fflush(None)
                os.dup2(saved, 1)
                os.close(saved)
            tmp.seek(0)
            lines = tmp.read().decode(errors="replace").splitlines()
        its = max([int(ln.split()[1].rstrip(":")) for ln in lines if ln.startswith("Iteration ")] or [0])
        return out, lines, its

    def solve(self, algorithm, Jt, mask, field=None, spacing=(1.0, 1.0, 1.0), **params):
        Jt = np.ascontiguousarray(Jt, dtype=self.dtype)
        nz, ny, nx = Jt.shape
        mask = np.ascontiguousarray(mask, dtype=np.bool_)
        out = (np.zeros((3, nz, ny, nx), self.dtype) if field is None
               else np.ascontiguousarray(field, dtype=self.dtype).copy())
        fn = {"gradient": lambda: self.lib.generate_displacement_gradient,
              "greedy": lambda: self.lib.generate_displacement_greedy,
              "matching": lambda: self.lib.volume_matching_3d}[algorithm]()
        fn(nx, ny, nz, *map(float, spacing), _ptr(Jt), _ptr(mask), *solver_params(**params),
           _ptr(out))
        if self.lib.disptools_has_error():
            raise RuntimeError("reference library reported an error")
        return out
