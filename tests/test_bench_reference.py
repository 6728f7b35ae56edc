"""CPU tests of bench.py's reference arm (the C restatement of the reference's FFTW path,
timed on the host): the JSON line the round-end comparison reads, on a small grid with a
short budget, and the silent exit of ranks other than 0 under torchrun."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env, *args):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env.update(extra_env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    r = run_bench({}, "--steps", "2", "--warmup", "3", "--grid", "128x96x64", "--ref-budget-s", "2")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    j = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in j, key
    assert j["impl"] == "reference" and j["unit"] == "Gpts/s" and j["higher_is_better"] is True
    assert j["steps"] == 2 and j["warmup"] == 3 and j["n_gpus"] == 1
    assert j["value"] > 0 and j["ms_per_step"] > 0 and j["dtype"] == "f64"
    assert j["config"]["nx"] == 128 and j["config"]["nz"] == 64 and 8 <= j["config"]["sample_ny"] <= 96
    cb = j["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == j["value"] and cb["sample"]
    assert j["e2e"] == {"value": j["value"], "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "2", "--warmup", "3",
                  "--grid", "128x96x64", "--ref-budget-s", "2")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
