"""Volume-parallel sharding of batched solves (host logic, CPU).

Two `gloo` ranks on this host split a batch of small volumes, solve their
shares with the oracle standing in for the device solver, and gather the
results; they must equal one local solve of every volume.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import pickle
import socket

import numpy as np
import pytest

from disptools_b200.sharding import assign_volumes


def test_assign_volumes_covers_each_volume_once():
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 4, 8):
        sizes = [int(v) for v in rng.integers(1, 1000, 37)]
        parts = assign_volumes(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        assert all(p == sorted(p) for p in parts)
        loads = [sum(sizes[i] for i in p) for p in parts]
        # longest-processing-time bound: no rank exceeds the mean by more
        # than one volume
        assert max(loads) <= sum(sizes) / world + max(sizes)


def test_assign_volumes_edge_cases():
    assert assign_volumes([], 3) == [[], [], []]
    assert assign_volumes([5], 3) == [[0], [], []]
    assert assign_volumes([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    assert assign_volumes([1, 9, 5], 2) == [[1], [0, 2]]
    with pytest.raises(ValueError):
        assign_volumes([1, 2], 0)
    with pytest.raises(ValueError):
        assign_volumes([-1], 2)


def _volumes():
    rng = np.random.default_rng(21)
    vols = []
    for shape in [(6, 7, 8), (9, 5, 6), (5, 5, 5), (8, 8, 7), (4, 6, 5)]:
        Jt = np.ascontiguousarray(1.0 + 0.05 * rng.standard_normal(shape))
        mask = np.ascontiguousarray(rng.random(shape) < 0.4)
        vols.append((Jt, mask))
    return vols


def _oracle_batched(vols, algorithm="gradient", precision="fp64", **params):
    from oracle.oracle import Oracle
    o = Oracle(4)
    out = []
    for v in vols:
        f, st = o.solve(algorithm, v[0], v[1], **params)
        out.append((f, {"iterations": st.iterations, "trials": st.trials, "reason": st.reason}))
    return out


def _child(rank, world, port, outdir):
    import torch.distributed as dist

    from disptools_b200.sharding import solve_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vols = _volumes()
        res_all = solve_sharded(vols, precision="fp64", gather="all", solve_fn=_oracle_batched,
                                it_max=15)
        res_root = solve_sharded(vols, precision="fp64", gather="root", solve_fn=_oracle_batched,
                                 it_max=15)
        res_mine = solve_sharded(vols, precision="fp64", gather="none", solve_fn=_oracle_batched,
                                 it_max=15)
        with open(os.path.join(outdir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump({"all": res_all, "root": res_root, "mine": res_mine}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_solve_sharded_two_gloo_ranks(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_child, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]

    vols = _volumes()
    expected = _oracle_batched(vols, it_max=15)
    parts = assign_volumes([v[0].size for v in vols], world)
    got = [pickle.load(open(tmp_path / f"rank{r}.pkl", "rb")) for r in range(world)]
    for r in range(world):
        assert len(got[r]["all"]) == len(vols)
        for (fe, se), (fg, sg) in zip(expected, got[r]["all"]):
            np.testing.assert_array_equal(fe, fg)
            assert se == sg
        assert sorted(got[r]["mine"]) == parts[r]
    assert got[1]["root"] is None
    for (fe, _), (fg, _) in zip(expected, got[0]["root"]):
        np.testing.assert_array_equal(fe, fg)
