"""bench.py's reference arm on the CPU: the reference's own CPU path (oracle/_ref) timed on
a small workload prints one JSON line with the contract's keys; under a multi-rank launch
only rank 0 prints. No GPU needed."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_ref_arm(env_extra):
    env = dict(os.environ, PYTHONPATH=ROOT, **env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "c1_8ves_p12", "--steps", "1", "--warmup", "0"], cwd=ROOT, env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line(ref):
    lines = run_ref_arm({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "vesicle-point velocity evaluations/s" and d["unit"] == "points/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "c1_8ves_p12" in d["config"]["workload"]


def test_reference_arm_other_ranks_print_nothing(ref):
    assert run_ref_arm({"WORLD_SIZE": "2", "RANK": "1"}) == []
