"""Volume-parallel batched solves over several GPUs, one process per GPU.

Independent volumes are the unit of work, as in the reference's Python
driver, which solves one volume per call (disptools/displacements.py:188-190).
The volumes of a batch are spread over the ranks of a process group by
voxel count.  Each rank runs one batched solve of its share on its own GPU,
and no collective runs during the solves.  One gather of the results
follows.

The assignment is longest-processing-time first:
* volumes are taken in decreasing voxel count (ties by index);
* each goes to the rank with the smallest load so far (ties: lowest rank).
It is a pure function of the sizes and the world size, so every rank computes
the same assignment without communication.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def assign_volumes(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the volumes each of `world` ranks solves (longest first,
    each to the least-loaded rank).  Every index appears exactly once; each
    rank's list is in increasing index order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    sizes = [int(s) for s in sizes]
    if any(s < 0 for s in sizes):
        raise ValueError("volume sizes must be non-negative")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def _voxels(volume) -> int:
    return int(np.prod(np.shape(volume[0])))


def solve_sharded(volumes: Sequence, algorithm: str = "gradient", precision: str = "mixed",
                  group=None, gather: str = "all", solve_fn: Callable | None = None, **params):
    """Solve a batch of independent host volumes across the ranks of `group`.

    ``volumes`` holds ``(J, mask[, field[, spacing]])`` tuples, as in
    :func:`disptools_b200.api.solve_batched`, on every rank.  This rank
    solves its share with ``solve_fn`` (default:
    :func:`disptools_b200.api.solve_batched` on the current device).

    ``gather``:
    * ``"all"`` returns every volume's ``(field, stats)`` on every rank;
    * ``"root"`` returns them on rank 0 only, and ``None`` elsewhere;
    * ``"none"`` returns this rank's own results, as a dict index -> result.

    Without an initialised process group this is one local batched solve.
    """
    if gather not in ("all", "root", "none"):
        raise ValueError("gather must be 'all', 'root' or 'none'")
    import torch.distributed as dist

    if solve_fn is None:
        from .api import solve_batched as solve_fn
    vols = list(volumes)
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if distributed else 1
    rank = dist.get_rank(group) if distributed else 0
    mine = assign_volumes([_voxels(v) for v in vols], world)[rank]
    results = solve_fn([vols[i] for i in mine], algorithm=algorithm, precision=precision,
                       **params) if mine else []
    local = dict(zip(mine, results))
    if gather == "none":
        return local
    if world == 1:
        return [local[i] for i in range(len(vols))]
    if gather == "all":
        parts = [None] * world
        dist.all_gather_object(parts, local, group=group)
    else:
        parts = [None] * world if rank == 0 else None
        dist.gather_object(local, parts, dst=0, group=group)
        if rank != 0:
            return None
    merged: dict = {}
    for p in parts:
        merged.update(p)
    if sorted(merged) != list(range(len(vols))):
        raise RuntimeError("the gathered results do not cover every volume exactly once")
    return [merged[i] for i in range(len(vols))]
