"""bench.py's reference arm on CPU: one JSON line with the contract's keys from
rank 0, nothing from the other ranks. (The GPU arm needs a device.)"""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_reference_arm(env_extra: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "3"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    done = run_reference_arm({"RANK": "0"})
    assert done.returncode == 0, done.stderr[-2000:]
    lines = [line for line in done.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["workload"] == "2d_type1_modes1024x1024_M1e7_uniform_eps1e-5"
    cpu = line["cpu_baseline"]
    assert cpu["kind"] in ("port", "reference") and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    assert cpu["unit"] == line["unit"] and cpu["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    done = run_reference_arm({"RANK": "1"})
    assert done.returncode == 0, done.stderr[-2000:]
    assert not [line for line in done.stdout.splitlines() if line.startswith("{")]
