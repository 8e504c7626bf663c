"""Build the native parts of disptools_b200 in-tree.

* ``libdisptools_b200.so`` — the CUDA library (sm_100a) with the C ABI of
  ``include/disptools_b200.h``;
* ``_disptools.<abi>.so`` — the NumPy extension with the method table of the
  reference ``_disptools`` module, linked against the library.

Run ``python disptools_b200/build.py`` (this file does not import the package,
which needs the built library).  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libdisptools_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                     f"-I{INCLUDE}", "-Xptxas", "-v"]

# (source, extra flags): the FP64 kernels and the matching solver (FP32, like
# its reference) are built without multiply-add contraction so their
# per-voxel arithmetic rounds like the reference C code.
UNITS = [
    ("dt_kernels_f32.cu", []),
    ("dt_kernels_f64.cu", ["-fmad=false"]),
    ("dt_capi.cu", []),
    ("dt_noalloc.cu", []),
    ("dt_resample.cu", []),
    ("dt_io.cpp", []),
    ("dt_maps.cu", []),
    ("dt_matching.cu", ["-fmad=false"]),
]
HEADERS = ["dt_internal.h", "dt_kernels.cuh", "dt_kernels_tma.cuh", "dt_tma.cuh"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], log: str | None = None) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log:
        with open(log, "w") as f:
            f.write(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd)}")


def build_library(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "disptools_b200.h")]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        stem = os.path.splitext(src)[0]
        o = os.path.join(BUILD, stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers, __file__]):
            _run([nvcc, *NVCC_FLAGS, *extra, "-c", s, "-o", o],
                 log=os.path.join(BUILD, stem + ".ptxas.txt"))
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-o", LIB, *objs])
    return LIB


def build_extension(force: bool = False) -> str:
    import numpy as np

    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(PKG, "_disptools" + suffix)
    src = os.path.join(PKG, "_disptools.c")
    if force or _stale(out, [src, LIB, os.path.join(INCLUDE, "disptools_b200.h")]):
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        _run([cc, "-std=c99", "-O2", "-fPIC", "-shared", "-Wall",
              f"-I{sysconfig.get_paths()['include']}", f"-I{np.get_include()}", f"-I{INCLUDE}",
              src, "-o", out, f"-L{PKG}", "-ldisptools_b200", "-Wl,-rpath,$ORIGIN"])
    return out


def build(force: bool = False) -> None:
    build_library(force)
    build_extension(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
