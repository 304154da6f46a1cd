"""The benchmark's reference arm on CPU: `bench.py --impl reference` times the
restated reference op on the host and prints one JSON line with the contract's
keys; under torchrun only rank 0 works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "solves/s"
    assert d["higher_is_better"] is True and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "screened_2048"
    # the GPU arm's config dict, key for key
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.workload_config(bench.make_instance(1), 1)
    # a step is one channel solve, and the line's time is the step's own
    ch = d["config"]["channels"]
    assert abs(d["ms_per_step"] * ch / 1e3 - 1.0 / d["value"]) <= 1e-9 / d["value"]
    assert d["solver"]["converged"] is True
    assert d["solver"]["sweeps_per_channel"][0] < d["config"]["max_iterations"]


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and not r.stdout.strip()
