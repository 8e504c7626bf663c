"""The benchmark's reference arm on this host (CPU): the reference C library
times the same workload and prints one JSON line with the contract's keys.
Small volumes keep the run short."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from oracle.oracle import Reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.skipif(not Reference.available("ref64"), reason="reference build not present")
@pytest.mark.parametrize("workload", ["c2", "greedy"])
def test_reference_arm_prints_one_contract_line(workload):
    d = _run("--workload", workload, "--size", "40", "--steps", "1", "--warmup", "0")
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "voxel-iters/s" and d["higher_is_better"] is True
    assert ("greedy" in d["metric"]) == (workload == "greedy")
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["size"] == [40, 40, 40]
