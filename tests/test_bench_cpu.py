"""bench.py's reference arm on the CPU (the oracle: the reference's CPU path restated in
C++): one JSON line with the contract's keys, and nothing from ranks other than 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


def test_reference_arm_json_line():
    r = _run({}, "--workload", "dam0", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "particle-updates/s"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == "dam0"


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--workload", "dam0", "--steps", "1",
             "--warmup", "0")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_on_the_batched_sample():
    r = _run({}, "--workload", "batched", "--scenes", "2", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["workload"] == "batched" and line["config"]["scenes"] == 2
