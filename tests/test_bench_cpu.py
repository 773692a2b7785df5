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


def test_reference_arm_loads_no_product_library():
    """The reference arm builds its scene with the oracle's lattice restatement: the
    process maps the oracle library and never the CUDA library of the product."""
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'dam0', '--steps', '1', "
            "'--warmup', '0']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPS', 'libvxl_sph' in maps, 'liboracle_wcsph' in maps)")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert "MAPS False True" in r.stdout, r.stdout[-500:]


def test_reference_arm_config_is_the_gpu_arms():
    """Both arms print the same `config` object for a plain workload."""
    r = _run({}, "--workload", "dam0", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    sys.path[:0] = [str(ROOT), str(ROOT / "rust-wl_b200")]
    import bench
    assert line["config"] == json.loads(json.dumps(bench.workload_config(bench.build_scene("dam0"))))


def test_gpus_flag_launches_ranks():
    """`--gpus 2` without a launcher starts two ranks itself (torch.distributed.run on
    127.0.0.1); on the reference arm rank 0 alone prints its line, with n_gpus 2."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "dam0", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"


def test_roofline_tables_point_at_committed_summaries():
    """roofline.traffic and roofline.issue come from committed ncu summaries: every row of
    the two tables parses and names a summary under profiles/, and the headline workload's
    dominant kernel has both figures."""
    sys.path.insert(0, str(ROOT))
    import bench
    for name, ncols in (("roofline_traffic.txt", 4), ("roofline_issue.txt", 5)):
        rows = [l.split() for l in (ROOT / "profiles" / name).read_text().splitlines()
                if l.strip() and not l.startswith("#")]
        assert rows, name
        for f in rows:
            assert len(f) == ncols, (name, f)
            float(f[2])
            assert (ROOT / "profiles" / f[-1]).is_file(), (name, f[-1])
    assert bench.ncu_traffic("k_density", "dam10m") > 0
    issue = bench.ncu_issue("k_density", "dam10m")
    assert 0.0 < issue["issue_active"] <= 1.0 and 0.0 < issue["threads_per_instruction"] <= 32.0
