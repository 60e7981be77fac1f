"""bench.py's reference arm (the oracle port timed on the host cores): one JSON
line with the keys the measurement contract names, on rank 0 only."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

KEYS = ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
        "cpu_baseline")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "3",
                           "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_prints_the_contract_line():
    out = _run({})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in KEYS:
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert (line["steps"], line["warmup"], line["n_gpus"]) == (3, 3, 1)
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["unit"] == line["unit"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["value"] == line["value"]
    assert cb["cores"] >= 1 and cb["sample"]
    assert "workload" in line["config"]
    # K + W small: every step is the full benchmark workload, and the config says so
    assert "4096x4096" in line["config"]["workload"] and line["config"]["cells_per_gpu"] == 4096 ** 2
    assert "full 4096x4096" in cb["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    out = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
