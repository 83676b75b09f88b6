"""bench.py's reference arm on the CPU: the JSON line's keys, the N>1 rule
(ranks other than 0 exit 0 without work or output), and that the time it
prints is whole frames that fit in the run's own wall time."""
import json
import os
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env):
    env = dict(os.environ)
    env.update(extra_env)
    t0 = time.perf_counter()
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    r.wall_s = time.perf_counter() - t0
    return r


def test_reference_arm_other_ranks_silent():
    r = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_json_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == "ms/frame" and d["unit"] == "ms/frame" and d["higher_is_better"] is False
    assert d["steps"] == 1 and d["warmup"] == 3 and d["value"] > 0
    # whole frames were timed: the claimed time fits in the process's own wall time
    assert (d["steps"] + d["warmup"]) * d["ms_per_step"] * 1e-3 <= r.wall_s
    assert "workload" in d["config"] and "model" not in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
