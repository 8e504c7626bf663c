"""Benchmark of the displacement-field generator (gradient method).

Workload (the headline configuration): a 256^3 volume, target J = clip(exp(
sum of 16 Gaussian blobs), 0.7, 1.4), mask = |log J| > 0.01 dilated by 3,
zero initial field, the reference's default parameters; FP32 field and
stencils with FP64 reductions.  One step = one solve from the zero field
capped at --it-max iterations.  Metric: voxel-iterations/s = voxels x
iterations completed / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank solves its own volume (independent volumes: weak
scaling, no collective on the data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "gradient-descent voxel-iters/s at 256³, FP32-mixed vs FP64 plain; % HBM peak"
UNIT = "voxel-iters/s"
# Algorithmic bytes per voxel of one launch (FP32 field): the trial reads the
# field, the gradient, the target map and the mask and writes the candidate;
# the gradient pass reads the field, the target map and the mask and writes
# the gradient.
BYTES_PER_VOXEL = {"trial": 12 + 12 + 4 + 1 + 12, "gradient": 12 + 4 + 1 + 12}
BYTES_PER_VOXEL_FP64 = {"trial": 24 + 24 + 8 + 1 + 24, "gradient": 24 + 8 + 1 + 24}
# Greedy method, per trial: the field, the target map and the mask in, the
# candidate out (the error map counted as recomputed in the tile).  This
# library streams the stored error map instead, 8 more bytes per voxel, which
# the traffic figure shows.
BYTES_PER_VOXEL_GREEDY = {"trial": 12 + 4 + 1 + 12}
METRIC_GREEDY = "greedy-method voxel-iters/s at 256³, FP32-mixed; % HBM peak"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--size", type=int, default=256)
    p.add_argument("--it-max", type=int, default=100)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-greedy", action="store_true")
    p.add_argument("--no-other-configs", action="store_true",
                   help="skip the short runs of configs 3, 4 and 5 that the default line carries")
    p.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5", "greedy", "matching"],
                   help="c2: one 256^3 volume per rank (default); c4: 64 volumes of "
                        "axes U{48..192} split over the ranks; c5: one 512x512x384 volume per "
                        "rank through a 3-level pyramid, plus greedy on the coarsest level; "
                        "greedy: the config-2 volume solved by the greedy method; "
                        "c3: the differentiable Jacobian, forward + backward, on 4 192x224x192 fields")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def iterations_done(st) -> int:
    # the loop counter exceeds it_max by one when the budget ran out
    return int(st["iterations"] - 1 if st["reason"] == "it_max" else st["iterations"])


def workload_c2(algorithm: str, n: int, it_max: int) -> str:
    """The workload string of the config-2 lines (both arms)."""
    return (f"config 2: {algorithm} method on {n}^3 (16 Gaussian blobs), zero initial field, "
            f"the reference's default parameters, it_max={it_max} per step")


def workload_matching(n: int, it_max: int) -> str:
    """The workload string of the matching lines (both arms)."""
    return (f"matching solver on {n}^3 (16 Gaussian blobs), zero initial field, the reference's default "
            f"parameters, it_max={it_max} per step")


MATCHING_SIZE = 128
MATCHING_SAMPLE_ITERATIONS = 10


def reference_impl():
    """The reference C library's FP64 build with its stock verbose output
    (what its Python package builds, setup.py: DISPTOOLS_VERBOSE=ON), which
    reports the iterations each solve completed; the restatement when the
    reference was not built."""
    from oracle.oracle import Oracle, Reference
    if Reference.available("ref64_verbose"):
        return Reference("ref64_verbose"), "reference"
    return Oracle(4), "port"


def reference_solve(impl, kind, algorithm, Jt, mask, it_max):
    """One solve from the zero field: (seconds, iterations completed, field)."""
    t0 = time.perf_counter()
    if kind == "reference":
        field, _, its = impl.solve_logged(algorithm, Jt, mask, it_max=it_max)
    else:
        field, st = impl.solve(algorithm, Jt, mask, it_max=it_max)
        its = st.iterations - 1 if st.reason == "it_max" else st.iterations
    return time.perf_counter() - t0, int(its), field


def reference_cpu_rate(Jt, mask, it_max, samples=3, warmup=1, algorithm="gradient"):
    """The reference C library (FP64, OpenMP, all host cores) solving the
    same volume with the same it_max: `warmup` short solves (it_max 2), then
    `samples` full ones.  Rate = voxels x iterations completed / time, summed
    over the samples; the last sample's field is returned for the accuracy
    comparison."""
    impl, kind = reference_impl()
    for _ in range(warmup):
        reference_solve(impl, kind, algorithm, Jt, mask, min(2, it_max))
    times, its, field = [], [], None
    for _ in range(samples):
        t, k, field = reference_solve(impl, kind, algorithm, Jt, mask, it_max)
        times.append(t)
        its.append(k)
    rate = Jt.size * sum(its) / sum(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return rate, kind, cores, times, its, field


def masked_residual(J, Jt, mask) -> float:
    """Final masked max |J - J_t| (the reference's max voxel error inside the
    mask, src/headers/error.h:87-172, without the tolerance band outside)."""
    import numpy as np
    d = np.abs(J - Jt)[mask]
    return float(d.max()) if d.size else 0.0


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    if args.workload == "c3":
        run_reference_c3(args)
        return
    if args.workload == "matching":
        run_reference_matching(args)
        return
    # the seeded generator only: this arm loads no library of this package
    from disptools_b200.synthetic import blob_problem
    n = args.size
    IT = args.it_max
    algorithm = "greedy" if args.workload == "greedy" else "gradient"
    Jt, mask = blob_problem((n, n, n), blobs=16, seed=0)
    impl, kind = reference_impl()
    # warm-up steps: short solves (threads and pages brought up)
    for _ in range(args.warmup):
        reference_solve(impl, kind, algorithm, Jt, mask, min(2, IT))
    times, its = [], []
    for _ in range(args.steps):
        t, k, _ = reference_solve(impl, kind, algorithm, Jt, mask, IT)
        times.append(t)
        its.append(k)
    value = Jt.size * sum(its) / sum(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"per step: one {algorithm} solve of the {n}^3 volume from the zero field, it_max={IT}, "
              f"reference C library (FLOAT_SIZE=64, ORDER_PD=4, OpenMP, verbose output as its "
              f"Python package builds it) through its C ABI; iterations per step {sorted(set(its))}")
    out = {
        "impl": "reference", "metric": METRIC_GREEDY if algorithm == "greedy" else METRIC, "value": value,
        "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": workload_c2(algorithm, n, IT), "size": [n, n, n], "it_max_per_step": IT,
                   "iterations_per_step": statistics.mean(its),
                   "warmup_steps": "it_max=2 solves"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def run_reference_matching(args):
    """The reference's volume_matching_3d (oracle/_ref, FP64 build, OpenMP)
    on the matching line's volume; each step a bounded sample of ten
    iterations of the same solve (the rate is per voxel-iteration)."""
    import ctypes as C

    from disptools_b200.synthetic import blob_problem
    from oracle.oracle import Reference
    n, IT = MATCHING_SIZE, args.it_max
    metric = "matching-solver voxel-iters/s, 128^3 (16 blobs)"
    if not Reference.available("ref64_match"):
        print(json.dumps({"impl": "reference", "metric": metric,
                          "unavailable": "the reference matching build (oracle/_ref) is missing"}))
        return
    # The reference's gradient reads malloc'd buffers it never clears
    # (src/VolumeMatching3D.c:422-427): perturb fills them with zeros.
    C.CDLL(None).mallopt(-6, 255)
    Jt, mask = blob_problem((n, n, n), blobs=16, seed=0)
    ref = Reference("ref64_match")
    k = min(IT, MATCHING_SAMPLE_ITERATIONS)
    for _ in range(args.warmup):
        ref.solve("matching", Jt, mask, it_max=1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.solve("matching", Jt, mask, it_max=k)
        times.append(time.perf_counter() - t0)
    value = Jt.size * k * len(times) / sum(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"per step: {k} iterations of the matching solve of the {n}^3 volume from the zero field "
              f"(a bounded sample of the it_max={IT} step), reference volume_matching_3d (OpenMP) through its "
              f"C ABI")
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_matching(n, IT), "iterations_per_step": k,
                   "warmup_steps": "it_max=1 solves"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_reference_c3(args):
    """The reference C library's jacobian_dynamic (FP64, OpenMP) on the
    config-3 fields.  The reference has no adjoint of its Jacobian, so a step
    is the forward map of the batch only; the line says so."""
    import numpy as np

    from disptools_b200.synthetic import smooth_field
    from oracle.oracle import Oracle, Reference
    shape, B = (192, 224, 192), 4
    fields = [smooth_field(shape, seed=b) for b in range(B)]
    impl, kind = (Reference("ref64"), "reference") if Reference.available("ref64") else (Oracle(4), "port")
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for f in fields:
            impl.jacobian(f)
        if s >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = statistics.mean(times)
    value = B * float(np.prod(shape)) / t
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    print(json.dumps({
        "impl": "reference",
        "metric": "differentiable jacobian() forward + backward voxels/s, 4 x 192x224x192 FP32 (config 3)",
        "value": value, "unit": "voxels/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "config 3 fields, forward map only (the reference has no adjoint)"},
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": cores, "kind": kind,
                         "sample": f"per step: jacobian_dynamic on 4 fields of {shape}"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_c4(args, world, rank, local, quiet=False):
    """Config 4: 64 independent volumes (axes U{48..192}, 1-4 ellipsoids
    each), FP32 fields.  The volumes are split over the ranks by voxel count
    (disptools_b200.sharding.assign_volumes) and each rank solves its share
    in one batched call per step: total work is fixed (strong scaling)."""
    import numpy as np
    import torch

    import disptools_b200 as dt
    from disptools_b200 import torch_ops
    from disptools_b200.sharding import assign_volumes
    from disptools_b200.synthetic import batch_sizes, ellipsoid_problem

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    IT = args.it_max
    sizes = batch_sizes(64, 48, 192, seed=0)
    total_vox = int(sum(np.prod(s) for s in sizes))
    mine = assign_volumes([int(np.prod(s)) for s in sizes], world)[rank]
    host = [ellipsoid_problem(sizes[i], seed=i) for i in mine]
    vols = [(torch.from_numpy(J).float().to(dev), torch.from_numpy(m).to(dev),
             torch.zeros((3,) + J.shape, dtype=torch.float32, device=dev)) for J, m in host]
    stream = torch.cuda.current_stream(dev)

    def step():
        for v in vols:
            v[2].zero_()
        return torch_ops.solve_batched(vols, it_max=IT) if vols else []

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = dt.kernel_launch_count()
    vi = 0.0
    trials = iters = 0
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            for (J, _, _), st in zip(vols, step()):
                k = iterations_done(st)
                vi += float(J.numel()) * k
                iters += k
                trials += st["trials"]
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    launches = dt.kernel_launch_count() - launches0
    tiles = dt.tile_config() if vols else None
    value = sum_over_ranks(world, vi) / (ms / 1000.0)

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        hv = [(pin(J), pin(m), pin(np.zeros((3,) + J.shape))) for J, m in host]
        dt.solve_batched(hv, it_max=IT, inplace=True)
        barrier(world)
        te = 0.0
        ve = 0.0
        ke = max(1, min(args.steps, 2))
        for _ in range(ke):
            for _, _, f in hv:
                f[...] = 0.0  # zero initial guess, written before the timed call
            t0 = time.perf_counter()
            res = dt.solve_batched(hv, it_max=IT, inplace=True) if hv else []
            te += time.perf_counter() - t0
            ve += sum(float(J.size) * iterations_done(st) for (J, _, _), (_, st) in zip(hv, res))
        te = max_over_ranks(world, te)
        nb = sum(J.nbytes + m.nbytes + f.nbytes for J, m, f in hv)
        e2e = {"value": sum_over_ranks(world, ve) / te, "unit": UNIT,
               "h2d_bytes_per_step": int(sum_over_ranks(world, nb)),
               "d2h_bytes_per_step": int(sum_over_ranks(world, sum(f.nbytes for _, _, f in hv))),
               "steps": ke, "path": "disptools_b200.solve_batched(inplace=True) (C ABI, host float64 "
                                     "arrays in pinned memory)"}

    line = {
        "metric": "batched gradient-descent voxel-iters/s, 64 volumes (config 4)",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"config 4: 64 volumes, axes U{{48..192}}, 1-4 ellipsoids, "
                               f"FP32 fields, it_max={IT} per step",
                   "voxels": total_vox, "volumes": len(sizes),
                   "l2": "inputs larger than L2 (fields of all volumes 1.5 GB)",
                   "iterations_per_step_rank0": iters / args.steps,
                   "trials_per_iteration_rank0": trials / max(iters, 1),
                   "parallelism": f"volumes split over {world} ranks by voxel count",
                   "tiles": tiles},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
}
    if rank == 0 and not quiet:
        print(json.dumps(line))
    return line


def run_c5(args, world, rank, local, quiet=False):
    """Config 5: a 512x512x384 volume (64 blobs as in config 2) per rank,
    FP32 fields.  One step = the 3-level pyramid of the gradient method
    (disptools_b200.pyramid.displacement, it_max per level = --it-max) on
    device tensors, then a greedy solve (it_max = --it-max) of the coarsest
    level's target.  Metric: voxel-iterations of all solves in the step
    (each level counted at its padded size) per second."""
    import numpy as np
    import torch

    import disptools_b200 as dt
    from disptools_b200 import pyramid, torch_ops
    from disptools_b200.synthetic import blob_problem_device

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    IT = args.it_max
    shape = (384, 512, 512)
    J, mask = blob_problem_device(shape, blobs=64, seed=rank, device=dev)
    sizes, spacings = pyramid.level_geometry(tuple(s + 2 for s in shape), (1.0, 1.0, 1.0), 3)
    # the coarsest level's target and mask for the greedy solve, built once
    Jp = torch.nn.functional.pad(J[None, None], (1,) * 6, mode="replicate")[0, 0]
    mp = torch.nn.functional.pad(mask.double()[None, None], (1,) * 6, mode="constant", value=0.0)[0, 0]
    Jc = pyramid.scale_image(Jp, spacings[0], sizes[2]).float().contiguous()
    mc = (pyramid.scale_image(mp, spacings[0], sizes[2], nearest=True) != 0).contiguous()
    fc = torch.zeros((3,) + sizes[2], dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        _, st = pyramid.displacement(J, mask=mask, levels=3, it_max=IT, return_stats=True)
        fc.zero_()
        sg = torch_ops.solve(Jc, mc, fc, spacing=spacings[2], algorithm="greedy", it_max=IT)
        vi = 0.0
        for s, size in zip(st, sizes[::-1]):
            vi += float(np.prod(size)) * iterations_done(s)
        vi += float(np.prod(sizes[2])) * iterations_done(sg)
        return vi, [iterations_done(s) for s in st] + [iterations_done(sg)]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = dt.kernel_launch_count()
    vi = 0.0
    its = None
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            v, its = step()
            vi += v
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    launches = dt.kernel_launch_count() - launches0
    value = sum_over_ranks(world, vi) / (ms / 1000.0)
    line = {
        "metric": "pyramid gradient-descent voxel-iters/s, 512x512x384 (config 5)",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"config 5: 512x512x384, 64 Gaussian blobs, 3-level pyramid "
                               f"(gradient, it_max={IT} per level) + greedy on the coarsest "
                               f"level (it_max={IT}), FP32 fields",
                   "level_sizes_padded": [list(s) for s in sizes],
                   "iterations_per_solve": its,
                   "l2": "inputs larger than L2 (finest field 1.2 GB)",
                   "parallelism": f"{world} independent volumes"},
        "gpu_launches": launches, "clocks": clk.summary(),
}
    if rank == 0 and not quiet:
        print(json.dumps(line))
    return line


def run_c3(args, world, rank, local, quiet=False):
    """Config 3: the differentiable Jacobian on a batch of 4 FP32 fields of
    192x224x192 per rank (smooth random fields, max |u| = 3).  One step = the
    forward map and the backward adjoint of torch_ops.jacobian for the batch.
    Metric: field voxels through forward + backward per second.  The roofline
    is the Jacobian kernel's, timed alone: 16 algorithmic bytes per voxel
    (field 12 in, J 4 out)."""
    import numpy as np
    import torch

    import disptools_b200 as dt
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import smooth_field

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shape, B = (192, 224, 192), 4
    f0 = torch.stack([torch.from_numpy(smooth_field(shape, seed=4 * rank + b)).float()
                      for b in range(B)]).to(dev)
    rng = np.random.default_rng(rank)
    w = torch.from_numpy(rng.standard_normal((B,) + shape)).float().to(dev)
    f = f0.clone().requires_grad_(True)
    nvox = B * int(np.prod(shape))
    stream = torch.cuda.current_stream(dev)

    def step():
        f.grad = None
        torch_ops.jacobian(f).backward(w)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = dt.kernel_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    launches = dt.kernel_launch_count() - launches0
    value = sum_over_ranks(world, float(nvox) * args.steps) / (ms / 1000.0)

    # Jacobian kernel alone (one launch per field), then the backward alone.
    def timed(fn, reps=10):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    # The two halves as the autograd step runs them: with the cofactor path
    # (the default for this layout) the forward also writes C = cof * ih
    # (36 B/voxel) and the backward is one gather of grad_J * C; otherwise
    # the forward writes the map only and the backward re-reads the field.
    fd = f.detach()
    J = torch.empty((B,) + shape, dtype=torch.float32, device=dev)
    G = torch.empty_like(fd)
    cof = torch_ops.uses_cofactor_path(fd)
    if cof:
        Cb = torch.empty((B, 9) + shape, dtype=torch.float32, device=dev)
        fwd_ms = timed(lambda: [torch_ops.jacobian_cof_raw(fd[b], out=J[b], cof=Cb[b]) for b in range(B)])
        bwd_ms = timed(lambda: [torch_ops.jacobian_adjoint_cof_raw(Cb[b], w[b], out=G[b]) for b in range(B)])
    else:
        fwd_ms = timed(lambda: [torch_ops.jacobian_raw(fd[b], out=J[b]) for b in range(B)])
        bwd_ms = timed(lambda: [torch_ops.jacobian_adjoint_raw(fd[b], w[b], out=G[b]) for b in range(B)])
    hbm, peak_kind = peaks()
    fwd_bpv = 52 if cof else 16  # field 12 in, map 4 (and C 36) out
    achieved = fwd_bpv * nvox / (fwd_ms / 1000.0) / 1e9
    traffic = None  # DRAM bytes of one launch (one field), from the committed ncu capture
    bwd_traffic = None  # the backward's passes, per field
    try:
        tj = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        if cof:
            traffic = tj["jacobian_cof_c3_field"]["bytes_per_launch"]
            bwd_traffic = tj["adjoint_cof_c3_field"]["gather_bytes_per_launch"]
        else:
            traffic = tj["jacobian_c3_field"]["bytes_per_launch"]
            bwd_traffic = tj["adjoint_c3_field"]["weight_pass_bytes_per_launch"] + tj["adjoint_c3_field"][
                "gather_bytes_per_launch"]
    except Exception:
        pass
    # The backward at the adjoint's algorithmic bytes: field 12 and gJ 4 in,
    # gradient 12 out per voxel (one fused pass would move just these).
    bwd_achieved = 28.0 * nvox / (bwd_ms / 1000.0) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import Oracle, Reference
        impl, kind = (Reference("ref64"), "reference") if Reference.available("ref64") else (Oracle(4), "port")
        f64 = fd[0].double().cpu().numpy()
        impl.jacobian(f64)
        t0 = time.perf_counter()
        impl.jacobian(f64)
        t = time.perf_counter() - t0
        cpu = {"value": np.prod(shape) / t, "unit": "voxels/s (forward map only)",
               "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)), "kind": kind,
               "sample": f"one {shape} field, reference jacobian_dynamic (FP64, OpenMP): {t:.3f} s"}
    line = {
        "metric": "differentiable jacobian() forward + backward voxels/s, 4 x 192x224x192 FP32 (config 3)",
        "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config 3: torch_ops.jacobian forward + backward on 4 FP32 fields of "
                               "192x224x192 (Gaussian-filtered noise, sigma 6, max |u| = 3)",
                   "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                   "l2": "inputs larger than L2 (fields 397 MB)",
                   "parallelism": f"{world} independent batches"},
        "roofline": {"bound": "hbm", "kernel": "k_jacobian_tma" + (" (map and C)" if cof else ""),
                     "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                     "peak_source": peak_kind, "bytes_per_voxel": fwd_bpv,
                     "bytes_per_launch": fwd_bpv * nvox // B, "avg_launch_ms": fwd_ms / B,
                     "backward": {"kernels": ("k_gather_tma (grad_J * C)" if cof
                                              else "k_jacobian_tma (weights) + k_gather_tma"),
                                  "bytes_per_voxel": 28,
                                  "achieved": bwd_achieved, "frac": bwd_achieved / hbm,
                                  "traffic_per_field": bwd_traffic, "ms_per_field": bwd_ms / B}},
        "cpu_baseline": cpu,
        "e2e": None,
        "gpu_launches": launches, "clocks": clk.summary(),
}
    if rank == 0 and not quiet:
        print(json.dumps(line))
    return line


def greedy_leg(dt, torch_ops, torch, Jt, mask, field, stream, IT, nvox, world):
    """The greedy method on the headline volume (same target, mask and
    it_max): device-timed solves, and its trial kernel's roofline at the 29
    algorithmic bytes per voxel of a greedy trial (field 12 + target 4 + mask
    1 in, candidate 12 out)."""
    def step():
        field.zero_()
        return torch_ops.solve(Jt, mask, field, algorithm="greedy", it_max=IT)

    dt.set_profiling(True)
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    dt.set_profiling(True)  # counters cleared
    k, iters = 3, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k):
        iters += iterations_done(step())
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = dt.kernel_profile()
    dt.set_profiling(False)
    hbm, peak_kind = peaks()
    nl, tot = prof.get("trial", (0, 0.0))
    avg = tot / max(nl, 1)
    bpl = BYTES_PER_VOXEL_GREEDY["trial"] * nvox
    achieved = bpl / (avg / 1000.0) / 1e9 if avg > 0 else 0.0
    traffic = None
    try:
        traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))["greedy_trial"][
            "bytes_per_launch_256"]
    except Exception:
        traffic = None
    value = nvox * iters / (ms / 1000.0)
    return {"metric": METRIC_GREEDY, "value": value, "unit": UNIT, "steps": k,
            "ms_per_step": ms / k, "iterations_per_step": iters / k,
            "roofline": {"bound": "hbm", "kernel": "greedy trial", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": peak_kind, "bytes_per_launch": bpl, "avg_launch_ms": avg,
                         "launches": nl}}


def run_matching(args, world, rank, local, quiet=False):
    """The matching solver (volume_matching_3d, src/VolumeMatching3D.c:408-557,
    on the device): a 128^3 volume of 16 Gaussian blobs (the config-2
    generator), zero initial field, it_max = --it-max per step.  `value`
    solves device-resident float64 tensors (dtb_volume_matching_device, the
    initial field zeroed on the device inside the step); `e2e` calls the C
    ABI (dtb_volume_matching) on pinned host float64 arrays, the zero initial
    guess written before each timed call, the copies inside.  The roofline is
    the gradient kernel's (28 algorithmic bytes per grid point: positions 12
    in, cell targets 4 in, step 12 out), timed by the library's profiling
    events over one further solve.  The CPU baseline is the reference's own
    volume_matching_3d on the same volume, ten iterations."""
    import ctypes as C

    import numpy as np
    import torch

    import disptools_b200 as dt
    from disptools_b200 import _native as N
    from disptools_b200 import torch_ops
    from disptools_b200.api import make_params
    from disptools_b200.synthetic import blob_problem

    torch.cuda.set_device(local)
    n, IT = MATCHING_SIZE, args.it_max
    Jt, mask = blob_problem((n, n, n), blobs=16, seed=rank)
    nvox = n ** 3
    dev = torch.device("cuda", local)
    Jd = torch.from_numpy(np.ascontiguousarray(Jt)).to(dev)
    md = torch.from_numpy(np.ascontiguousarray(mask)).to(dev)
    fd = torch.zeros((3, n, n, n), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    scrub = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # twice the L2

    def step():
        scrub.fill_(1)  # flush L2 between steps
        fd.zero_()
        return torch_ops.solve(Jd, md, fd, algorithm="matching", it_max=IT)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = dt.kernel_launch_count()
    barrier(world)
    iters = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            iters += step()["iterations"]
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    launches = dt.kernel_launch_count() - launches0
    value = sum_over_ranks(world, float(nvox) * iters) / (ms / 1000.0)

    # the gradient kernel's roofline: one more solve with profiling on
    dt.set_profiling(True)
    step()
    torch.cuda.synchronize()
    prof = dt.kernel_profile()
    dt.set_profiling(False)
    hbm, peak_kind = peaks()
    ng, tg = prof.get("match_gradient", (0, 0.0))
    nc, tc = prof.get("match_cost", (0, 0.0))
    avg = tg / max(ng, 1)
    bpl = 28 * nvox
    achieved = bpl / (avg / 1000.0) / 1e9 if avg > 0 else 0.0
    traffic = None
    try:
        traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))["match_gradient"][
            "bytes_per_launch_128"]
    except Exception:
        traffic = None
    roofline = {"bound": "hbm", "kernel": "matching gradient", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_kind, "bytes_per_launch": bpl,
                "avg_launch_ms": avg, "launches": ng,
                "cost_kernel": {"launches": nc, "avg_ms": tc / max(nc, 1)},
                "note": "issue-bound FP32 arithmetic (72 cofactors per cell under the reference's rounding); "
                        "the working set stays in L2"}

    # end to end through the C ABI on pinned host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        Jh = pin(np.ascontiguousarray(Jt))
        mh = pin(np.ascontiguousarray(mask))
        fh = pin(np.zeros((3, n, n, n)))
        prm = make_params(it_max=IT)
        stt = N.SolveStats()

        def e2e_step():
            fh[...] = 0.0
            t0 = time.perf_counter()
            rc = N.lib.dtb_volume_matching(n, n, n, 1.0, 1.0, 1.0, Jh.ctypes.data, mh.ctypes.data,
                                           C.byref(prm), fh.ctypes.data, C.byref(stt))
            dt_s = time.perf_counter() - t0
            N.check(rc)
            return stt.as_dict(), dt_s

        e2e_step()
        barrier(world)
        te, ie = 0.0, 0
        for _ in range(args.steps):
            st_e, dt_s = e2e_step()
            ie += st_e["iterations"]
            te += dt_s
        te = max_over_ranks(world, te)
        e2e = {"value": sum_over_ranks(world, float(nvox) * ie) / te, "unit": UNIT,
               "h2d_bytes_per_step": int(Jh.nbytes + fh.nbytes), "d2h_bytes_per_step": int(fh.nbytes),
               "steps": args.steps, "ms_per_step": te * 1000.0 / args.steps,
               "path": "dtb_volume_matching (C ABI, host float64 arrays in pinned memory; the mask is not "
                       "read, as by the reference)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import Reference
        if Reference.available("ref64_match"):
            # The reference's gradient reads malloc'd buffers it never clears
            # (src/VolumeMatching3D.c:422-427): perturb fills them with zeros.
            C.CDLL(None).mallopt(-6, 255)
            ref = Reference("ref64_match")
            t0 = time.perf_counter()
            ref.solve("matching", Jt, mask, it_max=MATCHING_SAMPLE_ITERATIONS)
            tcpu = time.perf_counter() - t0
            cpu = {"value": nvox * MATCHING_SAMPLE_ITERATIONS / tcpu, "unit": UNIT,
                   "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)), "kind": "reference",
                   "sample": f"reference volume_matching_3d (OpenMP) on the same volume, "
                             f"{MATCHING_SAMPLE_ITERATIONS} iterations: {tcpu:.2f} s"}
    line = {
        "metric": "matching-solver voxel-iters/s, 128^3 (16 blobs)", "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_matching(n, IT), "arrays": "device-resident float64",
                   "iterations_per_step": iters / args.steps, "parallelism": f"{world} independent volumes",
                   "l2": "flushed between steps (256 MB write); within a solve the working set (positions, "
                         "step and next positions, 25 MB each) stays in L2"},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches, "clocks": clk.summary(),
    }
    if rank == 0 and not quiet:
        print(json.dumps(line))
    return line


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.workload == "matching" and args.impl == "b200":
        run_matching(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "c5" and args.impl == "b200":
        run_c5(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "c3" and args.impl == "b200":
        run_c3(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "c4" and args.impl == "b200":
        run_c4(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import numpy as np
    import torch

    import disptools_b200 as dt
    from disptools_b200 import _native as N
    from disptools_b200 import torch_ops
    from disptools_b200.synthetic import blob_problem

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.size
    algorithm = "greedy" if args.workload == "greedy" else "gradient"
    bytes_per_voxel = BYTES_PER_VOXEL_GREEDY if algorithm == "greedy" else BYTES_PER_VOXEL
    Jt_np, mask_np = blob_problem((n, n, n), blobs=16, seed=rank)
    nvox = Jt_np.size
    IT = args.it_max

    Jt = torch.from_numpy(Jt_np).float().to(dev)
    mask = torch.from_numpy(mask_np).to(dev)
    field = torch.zeros((3, n, n, n), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        field.zero_()
        return torch_ops.solve(Jt, mask, field, algorithm=algorithm, it_max=IT)

    # Profiling adds event nodes to the step graphs: switch it on before the
    # warm-up so the profiled graphs are built there, not in the timed steps.
    dt.set_profiling(True)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs (counters cleared)
    dt.set_profiling(True)
    launches0 = dt.kernel_launch_count()
    iters = trials = 0
    solve_ms = []
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            st = step()
            iters += iterations_done(st)
            trials += st["trials"]
            solve_ms.append(st["device_ms"])
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    launches = dt.kernel_launch_count() - launches0
    # the gradient and greedy solvers' kernels (not the matching solver's)
    prof = {k: v for k, v in dt.kernel_profile().items() if k in ("trial", "gradient")}
    tiles = dt.tile_config()
    dt.set_profiling(False)
    field_mixed = field.double().cpu().numpy()  # the last timed solve's result
    ms_max = max_over_ranks(world, ms)
    total_vi = sum_over_ranks(world, float(nvox) * iters)
    value = total_vi / (ms_max / 1000.0)
    tbar = trials / max(iters, 1)

    # ---- roofline of the dominant kernel (device time of the launches that did work)
    hbm, peak_kind = peaks()
    dom = max(prof, key=lambda k: prof[k][1]) if prof else "trial"
    nl, tot_ms = prof.get(dom, (0, 0.0))
    avg_ms = tot_ms / max(nl, 1)
    bytes_launch = bytes_per_voxel[dom] * nvox
    achieved = bytes_launch / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            t = json.load(open(tpath))
            traffic = t.get("greedy_trial" if algorithm == "greedy" else dom, {}).get("bytes_per_launch_256")
        except Exception:
            traffic = None
    kernels = {k: {"launches": v[0], "avg_ms": v[1] / max(v[0], 1),
                   "achieved_gbs": bytes_per_voxel.get(k, 0) * nvox / (v[1] / max(v[0], 1) / 1000.0) / 1e9
                   if v[0] else None,
                   "share": v[1] / max(sum(x[1] for x in prof.values()), 1e-12)}
               for k, v in prof.items()}
    # Algorithmic bytes per voxel-iteration of the whole path: a gradient pass
    # and T trials (gradient method), or T trials (greedy method).
    path_bpv = 29 * tbar if algorithm == "greedy" else 29 + 41 * tbar
    path_achieved = path_bpv * value / 1e9 / world

    # ---- plain FP64 path (same workload, fewer steps)
    fp64 = None
    if not args.no_fp64:
        Jt64 = torch.from_numpy(Jt_np).to(dev)
        f64 = torch.zeros((3, n, n, n), dtype=torch.float64, device=dev)
        f64.zero_()
        torch_ops.solve(Jt64, mask, f64, algorithm=algorithm, it_max=IT)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it64 = 0
        k64 = max(1, min(args.steps, 2))
        for _ in range(k64):
            f64.zero_()
            s64 = torch_ops.solve(Jt64, mask, f64, algorithm=algorithm, it_max=IT)
            it64 += iterations_done(s64)
        torch.cuda.synchronize()
        t64 = time.perf_counter() - t0
        v64 = nvox * it64 / t64
        fp64 = {"value": v64, "unit": UNIT, "ratio_mixed_over_fp64": (value / world) / v64,
                "steps": k64}
        field_fp64 = f64.cpu().numpy()
        del Jt64, f64

    # ---- greedy method on the same volume (gradient workload only): its
    # trial kernel's roofline at 29 algorithmic bytes per voxel
    greedy = None
    if algorithm == "gradient" and not args.no_greedy:
        greedy = greedy_leg(dt, torch_ops, torch, Jt, mask, field, stream, IT, nvox, world)

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        from disptools_b200.api import make_params
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        Jh = pin(np.ascontiguousarray(Jt_np))
        mh = pin(np.ascontiguousarray(mask_np))
        fh = pin(np.zeros((3, n, n, n)))
        p = make_params(it_max=IT)
        stt = N.SolveStats()

        def e2e_step():
            """One C-ABI call on host buffers; returns (stats, seconds).  The
            zero initial guess is written before the timed call."""
            fh[...] = 0.0
            t0 = time.perf_counter()
            rc = N.lib.dtb_generate_displacement(N.algorithm_code(algorithm), 0, n, n, n, 1.0, 1.0, 1.0,
                                                 Jh.ctypes.data,
                                                 mh.ctypes.data, C.byref(p), fh.ctypes.data,
                                                 C.byref(stt))
            dt_s = time.perf_counter() - t0
            N.check(rc)
            return stt.as_dict(), dt_s

        e2e_step()
        barrier(world)
        te = 0.0
        ie = 0
        ke = max(1, min(args.steps, 3))
        for _ in range(ke):
            st_e, dt_s = e2e_step()
            ie += iterations_done(st_e)
            te += dt_s
        te = max_over_ranks(world, te)
        e2e = {"value": sum_over_ranks(world, float(nvox) * ie) / te, "unit": UNIT,
               "h2d_bytes_per_step": int(Jh.nbytes + mh.nbytes + fh.nbytes),
               "d2h_bytes_per_step": int(fh.nbytes), "steps": ke,
               "path": "dtb_generate_displacement (C ABI, host float64 arrays in pinned memory)"}

    # ---- CPU baseline (rank 0, N = 1 only): the reference solving the same
    # volume to the same it_max; its result is the FP64 oracle of `accuracy`
    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, times, its, field_ref = reference_cpu_rate(Jt_np, mask_np, IT, algorithm=algorithm)
        from oracle.oracle import Oracle, Reference
        fp32 = None
        if Reference.available("ref32_verbose"):
            r32 = Reference("ref32_verbose")
            reference_solve(r32, "reference", algorithm, Jt_np, mask_np, min(2, IT))
            t32, k32, _ = reference_solve(r32, "reference", algorithm, Jt_np, mask_np, IT)
            fp32 = {"value": nvox * k32 / t32,
                    "sample": f"the reference's default FP32 build (its Python package's), one solve with "
                              f"it_max={IT}: {k32} iterations in {t32:.2f} s"}
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "fp32_build": fp32,
               "sample": f"{n}^3 volume, {algorithm} method from the zero field, it_max={IT}: reference C "
                         f"library FP64 (OpenMP) through its C ABI, one warm-up solve (it_max=2), then "
                         f"{len(times)} solves of {its} iterations in "
                         f"{', '.join(f'{t:.2f}' for t in times)} s"}
        # Accuracy against the FP64 oracle: the final masked max |J - J_t| of
        # each result, its Jacobian recomputed in FP64 by the reference.
        ref = Reference("ref64") if Reference.available("ref64") else Oracle(4)
        r_ref = masked_residual(ref.jacobian(field_ref), Jt_np, mask_np)
        r_mix = masked_residual(ref.jacobian(field_mixed), Jt_np, mask_np)
        at_it_max = {"residual_mixed": r_mix, "residual_oracle": r_ref, "difference": abs(r_mix - r_ref),
                     "iterations_mixed": iters // max(args.steps, 1), "iterations_oracle": its[-1],
                     "oracle": f"reference C library FP64 ({kind}), same volume and it_max",
                     "note": "before convergence the mixed accept/reject sequence drifts from the FP64 one"}
        if fp64 is not None:
            at_it_max["fp64_field_max_abs_diff"] = float(np.max(np.abs(field_fp64 - field_ref)))
            at_it_max["residual_fp64"] = masked_residual(ref.jacobian(field_fp64), Jt_np, mask_np)
        accuracy = {"at_it_max": at_it_max, "converged": None}
        # The rule itself (final masked max |J - J_t| within 1e-4 of the FP64
        # oracle's) at the solver's own termination: the mixed solve to the
        # default it_max against the reference's converged run, summarised
        # in tests/golden/config2_converged.json (same volume, seed 0).
        cpath = os.path.join(ROOT, "tests", "golden", "config2_converged.json")
        if algorithm == "gradient" and n == 256 and rank == 0 and os.path.exists(cpath):
            cref = json.load(open(cpath))
            field.zero_()
            t0 = time.perf_counter()
            stc = torch_ops.solve(Jt, mask, field, algorithm="gradient", it_max=50000)
            tc = time.perf_counter() - t0
            r_conv = masked_residual(ref.jacobian(field.double().cpu().numpy()), Jt_np, mask_np)
            accuracy["converged"] = {
                "residual_mixed": r_conv, "residual_oracle": cref["masked_max"],
                "difference": abs(r_conv - cref["masked_max"]), "tolerance": 1e-4,
                "within_tolerance": abs(r_conv - cref["masked_max"]) <= 1e-4,
                "iterations_mixed": int(stc["iterations"]), "iterations_oracle": cref["iterations"],
                "stop_mixed": stc["reason"], "stop_oracle": cref["stop_line"], "mixed_solve_s": tc,
                "oracle": "reference C library FP64, default parameters, it_max 50000 "
                          "(tests/golden/config2_converged.json)"}

    # ---- short runs of configs 3, 4 and 5 (two timed steps each), so the
    # default line carries a number for every configuration.
    other = None
    if world == 1 and algorithm == "gradient" and n == 256 and not args.no_other_configs:
        sub = argparse.Namespace(**{**vars(args), "steps": 2, "warmup": 1, "no_e2e": True,
                                    "no_cpu_baseline": True})
        other = {}
        # Config 3's step is about 1 ms: ten timed steps after three warm-up
        # steps keep its figure off the launch latency of the first ones.
        sub_c3 = argparse.Namespace(**{**vars(sub), "steps": 10, "warmup": 3})
        for name, fn in (("c3", run_c3), ("c4", run_c4), ("c5", run_c5)):
            line = fn(sub_c3 if name == "c3" else sub, world, rank, local, quiet=True)
            other[name] = {k: line.get(k) for k in ("metric", "value", "unit", "ms_per_step", "steps", "warmup",
                                                    "roofline", "gpu_launches", "clocks")}
            other[name]["workload"] = line["config"]["workload"]
            if name == "c3":
                other[name]["forward_ms"] = line["config"]["forward_ms"]
                other[name]["backward_ms"] = line["config"]["backward_ms"]

    if rank == 0:
        out = {
            "metric": METRIC_GREEDY if algorithm == "greedy" else METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_c2(algorithm, n, IT),
                       "precision": "FP32 field and stencils, FP64 reductions and step control",
                       "size": [n, n, n], "it_max_per_step": IT,
                       "l2": "inputs larger than L2 (FP32 field 201 MB + "
                             + ("error map 67 MB + candidate 201 MB)" if algorithm == "greedy"
                                else "gradient 201 MB)"),
                       "iterations_per_step": iters / args.steps,
                       "trials_per_iteration": tbar, "parallelism": f"{world} independent volumes",
                       "tiles": tiles, "tiles_from": "autotuner (first solve of the shape, in warm-up)",
                       "solve_device_ms": [round(v, 3) for v in solve_ms]},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms,
                         "kernels": kernels,
                         "path_achieved_gbs": path_achieved,
                         "path_frac": path_achieved / hbm},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "fp64_plain": fp64,
            "accuracy": accuracy,
            "greedy": greedy,
            "other_configs": other,
        }
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
