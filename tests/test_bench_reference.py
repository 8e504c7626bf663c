"""The benchmark's reference arm on this host (CPU): the reference C library
times the same workload as the repository's arm (same workload string, same
it_max per step), prints one JSON line with the contract's keys, and maps no
library of this package.  Small volumes keep the run short."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from oracle.oracle import Reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Runs bench.py as __main__ in this interpreter, then reports on stderr
# whether the process mapped a shared library of this package.
_WRAP = (
    "import runpy, sys\n"
    "sys.argv = ['bench.py'] + sys.argv[1:]\n"
    "runpy.run_path('bench.py', run_name='__main__')\n"
    "maps = open('/proc/self/maps').read()\n"
    "bad = sorted({l.split()[-1] for l in maps.splitlines() if 'disptools_b200' in l})\n"
    "sys.stderr.write('PACKAGE_LIBS=' + repr(bad) + '\\n')\n")


def _run(*args):
    out = subprocess.run([sys.executable, "-c", _WRAP, "--impl", "reference", *args],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, out.stdout
    assert "PACKAGE_LIBS=[]" in out.stderr, out.stderr[-2000:]
    return json.loads(lines[0])


@pytest.mark.skipif(not Reference.available("ref64"), reason="reference build not present")
@pytest.mark.parametrize("workload", ["c2", "greedy"])
def test_reference_arm_prints_one_contract_line(workload):
    d = _run("--workload", workload, "--size", "40", "--it-max", "12", "--steps", "1", "--warmup", "1")
    sys.path.insert(0, ROOT)
    import bench
    algorithm = "greedy" if workload == "greedy" else "gradient"
    assert d["config"]["workload"] == bench.workload_c2(algorithm, 40, 12)
    assert d["config"]["it_max_per_step"] == 12
    assert 1 <= d["config"]["iterations_per_step"] <= 12
    assert abs(d["ms_per_step"] / 1000.0 - 40 ** 3 * d["config"]["iterations_per_step"] / d["value"]) \
        <= 0.05 * d["ms_per_step"] / 1000.0
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["unit"] == "voxel-iters/s" and d["higher_is_better"] is True
    assert ("greedy" in d["metric"]) == (workload == "greedy")
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["size"] == [40, 40, 40]


@pytest.mark.skipif(not Reference.available("ref64_match"), reason="reference matching build not present")
def test_reference_arm_matching_line():
    """The matching workload's reference arm: the reference's own
    volume_matching_3d, the b200 arm's workload string and metric."""
    d = _run("--workload", "matching", "--steps", "1", "--warmup", "1")
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == "matching-solver voxel-iters/s, 128^3 (16 blobs)"
    assert d["config"]["workload"] == bench.workload_matching(bench.MATCHING_SIZE, 100)
    assert d["config"]["iterations_per_step"] == bench.MATCHING_SAMPLE_ITERATIONS
    assert d["value"] > 0 and d["unit"] == "voxel-iters/s"
    assert abs(d["ms_per_step"] / 1000.0 - 128 ** 3 * 10 / d["value"]) <= 0.05 * d["ms_per_step"] / 1000.0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0
