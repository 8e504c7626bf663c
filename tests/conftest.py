"""Shared test set-up.

CPU tests (the default selection ``-m "not gpu"``) check the oracle against
the golden vectors and the reference build, the host-side logic of the C ABI
and the NumPy extension.  Tests marked ``gpu`` run the CUDA library on a
device and compare it with the oracle.
"""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def _ensure_built() -> None:
    """Build the oracle and (when stale) the CUDA library and extension.  The
    build script is loaded by path: importing the package needs the library."""
    import importlib.util
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"])
    spec = importlib.util.spec_from_file_location(
        "_dtb_build", os.path.join(ROOT, "disptools_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build()


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle(4)


@pytest.fixture(scope="session")
def oracle_pd2():
    from oracle.oracle import Oracle
    return Oracle(2)


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")
    return {
        "jacobian": dict(np.load(os.path.join(d, "jacobian.npz"))),
        "solver": dict(np.load(os.path.join(d, "solver.npz"))),
        "cases": json.load(open(os.path.join(d, "solver_cases.json"))),
    }
