"""Generate the golden fixtures of tests/golden/ from the reference C library.

The reference library (disptools v0.4.1, src/*.c) is compiled from its own
sources into oracle/_ref/ by oracle/Makefile (FLOAT_SIZE=64, ORDER_PD=4, and
ORDER_PD=2 for the gradient check).  This script calls it through its C ABI
(jacobian_dynamic, generate_displacement_gradient,
generate_displacement_greedy, and volume_matching_3d from
libdisptools_ref64_match) on seeded inputs and stores inputs and outputs
as small .npz files.  Run it where the reference sources are available:

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py --maps   # maps.npz only
    python tests/golden/make_golden.py --config2   # config2_converged.json (minutes)
    python tests/golden/make_golden.py --matching  # matching.npz only

maps.npz comes from the reference's own Python map functions
(disptools/displacements.py), executed from its source with the SimpleITK
calls answered by a small stand-in (the package needs SimpleITK, which is not
installed) and its _disptools calls by the reference C library.

Inputs are seeded synthetic data; the shapes mirror the reference's own tests
(test/test_displacements.py:43-55 uses sin_vector_field(10);
test/c/test_jacobian_macros.cpp:22-67 uses i*i data on a 5x6x7 grid with
spacing (2, 3, 4)).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference, build  # noqa: E402


def sin_vector_field(n: int) -> np.ndarray:
    """The field of disptools/drawing.py:368-390 in the library layout
    [3, z, y, x] (all three components equal)."""
    x = np.linspace(0, 0.5, n)
    xx, yy, zz = np.meshgrid(x, x, x)
    s = np.sin(xx ** 2 + yy ** 2 + zz ** 2)  # ITK array [z, y, x]
    return np.ascontiguousarray(np.stack([s, s, s]))


def i2_field() -> np.ndarray:
    """data[i] = i*i over a 3 x 7 x 6 x 5 buffer (test_jacobian_macros.cpp:53-59)."""
    nx, ny, nz = 5, 6, 7
    i = np.arange(3 * nz * ny * nx, dtype=np.float64)
    return (i * i).reshape(3, nz, ny, nx)


def ball(n, c, r):
    z, y, x = np.meshgrid(*[np.arange(n)] * 3, indexing="ij")
    return (x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 <= r * r


def small_problem(seed: int, shape):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    Jt = np.ones(shape)
    mask = np.zeros(shape, bool)
    for _ in range(2):
        c = rng.uniform([2, 2, 2], [nz - 3, ny - 3, nx - 3])
        r = rng.uniform(1.5, 3.0)
        inside = (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 <= r * r
        Jt[inside] = rng.uniform(0.85, 1.15)
        mask |= (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 <= (r + 1) ** 2
    return np.ascontiguousarray(Jt), np.ascontiguousarray(mask)


class _Image:
    """The part of a SimpleITK image that the reference's map functions use:
    the pixel array ([z, y, x] or [z, y, x, 3]), spacing, CopyInformation."""

    def __init__(self, arr, spacing=(1.0, 1.0, 1.0)):
        self.arr = np.asarray(arr)
        self.spacing = tuple(spacing)

    def GetSize(self):
        return tuple(reversed(self.arr.shape[:3]))

    def GetSpacing(self):
        return self.spacing

    def CopyInformation(self, other):
        self.spacing = other.spacing


def _sitk_stub(files):
    """SimpleITK calls of disptools/displacements.py:23-95 and :486-668 on
    _Image objects; `files` maps file names to images (ReadImage).
    Threshold follows ITK's ThresholdImageFilter with ThresholdOutside:
    values outside [lower, upper] (NaN included) become outsideValue."""
    import types
    st = types.SimpleNamespace()
    st.Cast = lambda img, t: _Image(np.asarray(img.arr, dtype=np.float64), img.spacing)
    st.GetArrayViewFromImage = lambda img: img.arr
    st.GetArrayFromImage = lambda img: np.array(img.arr, copy=True)
    st.GetImageFromArray = lambda a, isVector=False: _Image(np.array(a, copy=True))
    st.Image = lambda img: _Image(np.array(img.arr, copy=True), img.spacing)
    st.ReadImage = lambda f: files[f]
    st.Threshold = lambda img, lower, upper, outsideValue: _Image(
        np.where((img.arr >= lower) & (img.arr <= upper), img.arr, outsideValue), img.spacing)
    return st


def reference_map_functions(ref, files):
    """regularise, jacobian, jacobian_to_volume_change, average_jacobian and
    average_jacobian_from_displacements, executed from the reference's own
    source (disptools/displacements.py; extracted with ast, since the package
    imports SimpleITK, which is not installed).  Their SimpleITK calls go to
    _sitk_stub, their _disptools calls to the reference C library `ref`."""
    import ast
    import fnmatch
    import logging
    import re
    import types
    from oracle.oracle import reference_dir
    path = os.path.join(reference_dir(), "disptools", "displacements.py")
    tree = ast.parse(open(path).read(), path)
    names = {"regularise", "jacobian", "jacobian_to_volume_change", "average_jacobian",
             "average_jacobian_from_displacements"}
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    assert {n.name for n in body} == names, "reference functions not found"
    for n in body:  # annotations name sitk types; not evaluated
        n.returns = None
        for a in n.args.args:
            a.annotation = None

    def c_jacobian(spacing, field, out):
        out[...] = ref.jacobian(field, spacing)

    def c_regularise(arr, eps):
        arr[...] = ref.regularise(arr, eps)

    ns = {
        "np": np, "sitk": _sitk_stub(files), "logging": logging, "re": re,
        "glob": lambda pat: sorted(f for f in files if fnmatch.fnmatch(f, pat)),
        "_disptools": types.SimpleNamespace(jacobian=c_jacobian, regularise=c_regularise),
        "io": types.SimpleNamespace(read_rvf=lambda f: files[f]),
        "np_float_type": np.float64, "sitk_float_type": None, "sitk_vector_float_type": None,
    }
    exec(compile(ast.Module(body=body, type_ignores=[]), path, "exec"), ns)
    return ns


def map_fixtures(ref) -> dict:
    """Golden vectors of the Jacobian-map utilities (disptools/displacements.py:
    486-668) and of regularise (src/jacobian.c:29-55), from the reference's
    own code on seeded maps and fields."""
    rng = np.random.default_rng(7)
    out = {}
    shape = (9, 11, 13)
    maps = []
    for k in range(4):
        J = rng.uniform(-0.2, 2.5, shape)
        J.flat[:5] = [0.0, 1e-6, 1.0, 2e9, 1e-5]
        maps.append(J)
        out[f"map{k}"] = J
    fields = [rng.normal(scale=0.3, size=(3, 8, 9, 10)) for _ in range(3)]
    spacing = (0.9, 1.1, 1.3)
    files = {f"j{k}.vtk": _Image(m) for k, m in enumerate(maps)}
    # vector images: pixel arrays [z, y, x, 3]
    files.update({f"u{k}.rvf": _Image(np.moveaxis(f, 0, -1).copy(), spacing) for k, f in enumerate(fields)})
    for k, f in enumerate(fields):
        out[f"field{k}"] = f
    out["spacing"] = np.array(spacing)
    R = reference_map_functions(ref, files)
    for eps in (1e-5, 0.3):
        tag = str(eps).replace(".", "p").replace("-", "m")
        out[f"volume_change_{tag}"] = R["jacobian_to_volume_change"](_Image(maps[0].copy()), eps).arr
        out[f"average_jacobian_{tag}"] = R["average_jacobian"]("j*.vtk", eps).arr
        out[f"average_from_fields_{tag}"] = R["average_jacobian_from_displacements"]("u*.rvf", eps).arr
    # regularise with NaN and infinities (src/jacobian.c:29-55: J < eps -> eps)
    Jr = maps[1].copy()
    Jr.flat[5:9] = [np.nan, -np.inf, np.inf, -0.0]
    out["regularise_in"] = Jr
    out["regularise_out_0p05"] = R["regularise"](_Image(Jr.copy()), 0.05).arr
    return out


def config2_converged(ref_verbose) -> dict:
    """The headline volume (config 2: 256^3, 16 Gaussian blobs, seed 0) solved
    by the reference C library (FP64, verbose build) from the zero field with
    the default parameters and it_max 50000 (the reference wrapper's), i.e.
    to its own termination.  Stored as a summary: iterations, the last
    printed line, the final masked max |J - J_t| of the returned field
    (recomputed by the reference's jacobian), the field's sums and one line."""
    from disptools_b200.synthetic import blob_problem
    Jt, mask = blob_problem((256, 256, 256), blobs=16, seed=0)
    field, lines, its = ref_verbose.solve_logged("gradient", Jt, mask, it_max=50000)
    J = Reference("ref64").jacobian(field)
    last = [ln for ln in lines if ln.startswith("Iteration")][-1].split()
    return {
        "iterations": its,
        "stop_line": lines[-1],
        "total_error": float(last[4]),
        "max_voxel_error": float(last[8]),
        "masked_max": float(np.max(np.abs(J - Jt)[mask])),
        "field_abs_sum": float(np.abs(field).sum()),
        "field_line": field[:, 128, 128, ::8].tolist(),
        "threads": os.environ.get("OMP_NUM_THREADS", str(os.cpu_count())),
    }


def matching_fixtures() -> dict:
    # Matching solver (src/VolumeMatching3D.c), FP32 arithmetic.  Its first
    # gradient accumulates into malloc'd buffers it never clears
    # (src/VolumeMatching3D.c:422-427 and :445): with whatever the allocator
    # hands back its results are NaN or depend on earlier allocations.  This
    # script therefore runs with MALLOC_PERTURB_=255 (see main), under which
    # glibc fills every malloc'd block with zero bytes, i.e. the buffers
    # start cleared, as every later gradient of the reference does.
    refm = Reference("ref64_match")
    mat = {}
    for k, (shape, init, spacing, it_max) in enumerate([
        ((20, 20, 20), False, (1.0, 1.0, 1.0), 60),
        ((14, 12, 10), True, (1.0, 1.0, 1.0), 40),
        ((12, 13, 11), False, (0.8, 1.1, 1.25), 40),
        # several tiles along every axis of the device kernels, the last
        # tile of each axis one point wider than the others
        ((9, 17, 65), True, (1.0, 0.9, 1.2), 12),
    ]):
        if k == 0:
            mask = ball(20, 10, 5)
            Jt = np.where(mask, 1.1, 1.0)
        else:
            Jt, mask = small_problem(300 + k, shape)
        field0 = (np.random.default_rng(400 + k).normal(scale=0.05, size=(3,) + shape)
                  if init else np.zeros((3,) + shape))
        out = refm.solve("matching", Jt, mask, field=field0, spacing=spacing, it_max=it_max)
        mat[f"m{k}_Jt"] = Jt
        mat[f"m{k}_mask"] = mask
        mat[f"m{k}_field0"] = field0
        mat[f"m{k}_spacing"] = np.array(spacing)
        mat[f"m{k}_it_max"] = np.array(it_max)
        mat[f"m{k}_out"] = out
    return mat


def matching_pyramid_fixture() -> dict:
    # The multi-resolution wrapper (disptools/displacements.py:238-480, as
    # restated in oracle/pyramid.py) with the reference's matching solver at
    # every level: two levels, one voxel of padding, anisotropic spacing.
    from oracle import pyramid as P
    Jt, mask = small_problem(330, (18, 20, 22))
    kw = dict(levels=2, it_max=[15, 15], spacing=(1.0, 1.1, 0.9))
    out = P.displacement(Jt, mask=mask, algorithm="matching", solver=Reference("ref64_match"), **kw)
    return {"Jt": Jt, "mask": mask, "spacing": np.array(kw["spacing"]), "it_max": np.array(kw["it_max"]),
            "levels": np.array(kw["levels"]), "out": out}


def main() -> None:
    if "--config2" in sys.argv:
        build(ref=True)
        out = config2_converged(Reference("ref64_verbose"))
        with open(os.path.join(HERE, "config2_converged.json"), "w") as fh:
            json.dump(out, fh, indent=1)
        print("config-2 summary written to", HERE)
        return
    if "--maps" in sys.argv:
        build(ref=True)
        np.savez_compressed(os.path.join(HERE, "maps.npz"), **map_fixtures(Reference("ref64")))
        print("map fixtures written to", HERE)
        return
    if os.environ.get("MALLOC_PERTURB_") != "255":
        # zero-filled mallocs for the reference matching solver (see below)
        os.execve(sys.executable, [sys.executable, os.path.abspath(__file__)] + sys.argv[1:],
                  {**os.environ, "MALLOC_PERTURB_": "255"})
    build(ref=True)
    if "--matching" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "matching.npz"), **matching_fixtures())
        np.savez_compressed(os.path.join(HERE, "matching_pyramid.npz"), **matching_pyramid_fixture())
        print("matching fixtures written to", HERE)
        return
    ref = Reference("ref64")
    ref2 = Reference("ref64_pd2")

    # Jacobian fixtures ---------------------------------------------------
    rng = np.random.default_rng(0)
    jac = {}
    f = sin_vector_field(10)
    jac["sin10_field"] = f
    jac["sin10_J"] = ref.jacobian(f, (1.0, 1.0, 1.0))
    f = i2_field()
    jac["i2_field"] = f
    jac["i2_J"] = ref.jacobian(f, (2.0, 3.0, 4.0))
    for k, shape in enumerate([(3, 3, 3), (4, 5, 6), (7, 9, 11), (12, 5, 3)]):
        f = rng.normal(scale=0.3, size=(3,) + shape)
        sp = tuple(rng.uniform(0.5, 2.0, 3))
        jac[f"rand{k}_field"] = f
        jac[f"rand{k}_spacing"] = np.array(sp)
        jac[f"rand{k}_J"] = ref.jacobian(f, sp)
        jac[f"rand{k}_J_pd2"] = ref2.jacobian(f, sp)
    np.savez_compressed(os.path.join(HERE, "jacobian.npz"), **jac)

    # Solver fixtures (small volumes, full fields) ------------------------
    sol = {}
    cases = []
    for k, (alg, shape, init, extra) in enumerate([
        ("gradient", (12, 11, 10), False, {}),
        ("gradient", (9, 13, 8), True, {"strict": True}),
        ("gradient", (10, 10, 10), False, {"zeta": 100.0, "eta_max": 2.0}),
        ("greedy", (12, 11, 10), False, {}),
        ("greedy", (9, 13, 8), True, {}),
    ]):
        Jt, mask = small_problem(100 + k, shape)
        field0 = (np.random.default_rng(200 + k).normal(scale=0.05, size=(3,) + shape)
                  if init else np.zeros((3,) + shape))
        params = dict(it_max=200, **extra)
        out = ref.solve(alg, Jt, mask, field=field0, spacing=(1.0, 1.1, 0.9), **params)
        sol[f"c{k}_Jt"] = Jt
        sol[f"c{k}_mask"] = mask
        sol[f"c{k}_field0"] = field0
        sol[f"c{k}_out"] = out
        cases.append({"name": f"c{k}", "algorithm": alg, "spacing": [1.0, 1.1, 0.9],
                      "params": params})
    np.savez_compressed(os.path.join(HERE, "solver.npz"), **sol)

    # Config 1 (40^3 sphere): summary of the reference result -------------
    n = 40
    m = ball(n, 20, 10)
    Jt = np.where(m, 1.1, 1.0)
    out = ref.solve("gradient", Jt, m, it_max=1000)
    Jout = ref.jacobian(out)
    c1 = {
        "masked_max": float(np.max(np.abs(Jout - Jt)[m])),
        "total_error": float(np.sum(np.where(m, Jout - Jt, np.where(np.abs(Jout - Jt) < 0.2, 0.0,
                                                                      np.sign(Jout - Jt) * (np.abs(Jout - Jt) - 0.2))) ** 2)),
        "field_l2": float(np.sqrt(np.sum(out ** 2))),
        "field_line": out[:, 20, 20, :].tolist(),
    }
    with open(os.path.join(HERE, "solver_cases.json"), "w") as fh:
        json.dump({"cases": cases, "config1": c1}, fh, indent=1)

    mat = matching_fixtures()
    np.savez_compressed(os.path.join(HERE, "matching.npz"), **mat)
    np.savez_compressed(os.path.join(HERE, "matching_pyramid.npz"), **matching_pyramid_fixture())
    np.savez_compressed(os.path.join(HERE, "maps.npz"), **map_fixtures(ref))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
