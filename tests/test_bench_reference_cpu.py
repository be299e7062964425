"""bench.py --impl reference on the CPU: the reference arm's JSON line.

The reference arm times the reference's CPU path (the oracle port, compiled
with the reference's flags) on our arm's workload and metric; under torchrun
only rank 0 runs and prints.  This runs the real command (about half a minute
on 8 cores) and checks the line's contract.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    env.pop("CUDA_VISIBLE_DEVICES", None)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           *args], capture_output=True, text=True, cwd=ROOT, env=env, timeout=900)


def test_reference_arm_line():
    p = _run({}, "--steps", "1", "--warmup", "0")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"]["workload"] == bench.WORKLOAD
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["cores"] >= 1 and "GHMATECD" in cb["sample"] and "ZGESV" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "1", "--warmup", "0")
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
