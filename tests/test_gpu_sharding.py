"""Volume-parallel sharding through the device solver (GPU).

Two `gloo` ranks, each a process of its own on the same GPU, split a batch
of volumes, solve their shares with the library's batched device solver
(FP64) and gather the results.  The solves are independent (no kernel of
one rank waits for the other's), so the ranks may share the device.  The
gathered fields must equal one batched solve of every volume in a single
process, bit for bit.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import pickle
import socket

import numpy as np
import pytest

from disptools_b200.sharding import assign_volumes

pytestmark = pytest.mark.gpu


def _volumes():
    rng = np.random.default_rng(31)
    vols = []
    for shape in [(24, 20, 18), (12, 30, 16), (33, 9, 14), (16, 16, 16), (10, 12, 40)]:
        Jt = np.ascontiguousarray(1.0 + 0.08 * rng.standard_normal(shape))
        mask = np.ascontiguousarray(rng.random(shape) < 0.4)
        vols.append((Jt, mask))
    return vols


def _child(rank, world, port, outdir):
    import torch.distributed as dist

    from disptools_b200.sharding import solve_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = solve_sharded(_volumes(), precision="fp64", gather="all", it_max=30)
        mine = solve_sharded(_volumes(), precision="fp64", gather="none", it_max=30)
        with open(os.path.join(outdir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump({"all": [(fld, st["iterations"], st["trials"], st["reason"]) for fld, st in res],
                         "mine": sorted(mine)}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_solve_sharded_device_two_ranks_one_gpu(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_child, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]

    import disptools_b200 as dt
    vols = _volumes()
    expected = dt.solve_batched(vols, precision="fp64", it_max=30)
    parts = assign_volumes([v[0].size for v in vols], world)
    for r in range(world):
        got = pickle.load(open(tmp_path / f"rank{r}.pkl", "rb"))
        assert got["mine"] == parts[r]
        assert len(got["all"]) == len(vols)
        for (fe, se), (fg, it, tr, reason) in zip(expected, got["all"]):
            np.testing.assert_array_equal(fe, fg)
            assert (se["iterations"], se["trials"], se["reason"]) == (it, tr, reason)
