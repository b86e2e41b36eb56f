"""The benchmark's reference arm (CPU, no GPU needed): one JSON line with the GPU
arm's metric, unit, direction and workload description, the number of steps it
actually timed, and its CPU baseline and e2e objects."""

from __future__ import annotations

import argparse
import json
import subprocess
import sys

from conftest import REPO


def test_reference_arm_prints_the_contract_line():
    import bench

    cmd = [sys.executable, "bench.py", "--impl", "reference", "--steps", "3", "--warmup", "1",
           "--rows", "96", "--cols", "128"]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "cell-updates/s"
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["steps"] == 3 and line["warmup"] == 1
    # the GPU arm prints the same workload description for the same arguments
    args = argparse.Namespace(rows=96, cols=128, spinup=200)
    assert line["config"] == bench._config(args, 1)
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
