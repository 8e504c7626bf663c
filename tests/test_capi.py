"""The C-ABI library loads and exports every declared symbol; host-side
argument checking and the error state work without a GPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "disptools_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and not n.isupper()})


def test_library_exports_every_declared_symbol():
    from disptools_b200 import _native as N
    names = declared_functions()
    assert "generate_displacement_gradient_cuda" in names and len(names) >= 15
    for n in names:
        assert hasattr(N.lib, n), n
    assert set(names) == set(N.EXPORTED)


def test_float_type_size_and_error_state():
    from disptools_b200 import _native as N
    assert N.lib.get_float_type_size() == 64
    N.lib.disptools_clear_error()
    assert not N.lib.disptools_has_error()
    err = N.lib.disptools_get_error().contents
    assert err.line == -1 and err.message == b""


def _solve_rc(nx=3, ny=3, nz=3, **params):
    from disptools_b200 import _native as N
    from disptools_b200.api import make_params
    J = np.ones((nz, ny, nx))
    m = np.ones((nz, ny, nx), bool)
    f = np.zeros((3, nz, ny, nx))
    p = make_params(**params)
    return N.lib.dtb_generate_displacement(0, 0, nx, ny, nz, 1.0, 1.0, 1.0, J.ctypes.data,
                                           m.ctypes.data, C.byref(p), f.ctypes.data, None)


def test_rejects_too_small_volumes():
    from disptools_b200 import _native as N
    assert _solve_rc(nx=2) == N.ERR_ARGUMENT
    assert N.lib.disptools_has_error()
    assert b"at least 3" in N.lib.disptools_get_error().contents.message


@pytest.mark.parametrize("bad", [dict(alpha=0.0), dict(beta=-1.0), dict(epsilon=0.0),
                                 dict(eta=0.0), dict(theta=-1e-3), dict(it_max=-1)])
def test_rejects_invalid_parameters(bad):
    """ASSERT_PARAMETERS (src/headers/disptools.h:107-152) as errors."""
    from disptools_b200 import _native as N
    assert _solve_rc(5, 5, 5, **bad) == N.ERR_ARGUMENT
    assert N.lib.disptools_has_error()


def test_invalid_algorithm_and_precision():
    from disptools_b200 import _native as N
    from disptools_b200.api import make_params
    p = make_params()
    J = np.ones((4, 4, 4)); m = np.ones((4, 4, 4), bool); f = np.zeros((3, 4, 4, 4))
    rc = N.lib.dtb_generate_displacement(7, 0, 4, 4, 4, 1.0, 1.0, 1.0, J.ctypes.data, m.ctypes.data,
                                         C.byref(p), f.ctypes.data, None)
    assert rc == N.ERR_ARGUMENT
    rc = N.lib.dtb_generate_displacement(0, 9, 4, 4, 4, 1.0, 1.0, 1.0, J.ctypes.data, m.ctypes.data,
                                         C.byref(p), f.ctypes.data, None)
    assert rc == N.ERR_ARGUMENT
    assert N.lib.dtb_set_default_precision(5) == N.ERR_ARGUMENT
    assert N.lib.dtb_get_default_precision() in (0, 1)


def test_python_api_argument_checks():
    import disptools_b200 as dt
    with pytest.raises(TypeError):
        dt.solve(np.ones((4, 4, 4), np.float32), np.ones((4, 4, 4), bool))
    with pytest.raises(TypeError):
        dt.solve(np.ones((4, 4, 4)), np.ones((4, 4, 4), np.uint8))
    with pytest.raises(ValueError):
        dt.solve(np.ones((4, 4, 4)), np.ones((4, 4, 5), bool))
    with pytest.raises(ValueError):
        dt.solve(np.ones((4, 4, 4)), np.ones((4, 4, 4), bool), algorithm="bogus")
    with pytest.raises(ValueError):  # matching needs two voxels per axis
        dt.solve(np.ones((1, 4, 4)), np.ones((1, 4, 4), bool), algorithm="matching")
    with pytest.raises(ValueError):
        dt.solve(np.ones((4, 4, 4)), np.ones((4, 4, 4), bool), algorithm="matching", zeta=-1.0)
    with pytest.raises(TypeError):
        dt.solve(np.ones((4, 4, 4)), np.ones((4, 4, 4), bool), bogus=1)
