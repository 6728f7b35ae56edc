"""bench.py's engine arm on a small grid: one JSON line with every key of the contract
(roofline, e2e through the host-buffer call, clocks, launch count, the CPU baseline and
the parity of the measured step against the oracle in both band modes)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_engine_arm_prints_the_contract_line(cuda_device):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "4", "--warmup", "3",
                        "--no-extra", "--e2e-steps", "1", "--grid", "128x96x64",
                        "--rough-grid", ""], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    j = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "clocks", "gpu_launches"):
        assert key in j, key
    assert j["n_gpus"] == 1 and j["steps"] == 4 and j["warmup"] == 3 and j["unit"] == "Gpts/s"
    assert j["value"] > 0 and j["ms_per_step"] > 0 and j["higher_is_better"] is True
    assert j["gpu_launches"] >= 4 * 4
    roof = j["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in roof, key
    assert roof["achieved"] > 0 and roof["peak"] > 0 and roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"])
    e2e = j["e2e"]
    nh = 130 * 66 * 98
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] == 3 * 8 * nh
    assert e2e["d2h_bytes_per_step"] == 3 * 8 * nh + 8 * 128 * 96 * 64
    assert "sm_mhz" in j["clocks"] and "reasons" in j["clocks"]
    cpu = j["cpu_baseline"]
    assert cpu["value"] > 0 and cpu["kind"] == "port" and cpu["cores"] >= 1
    acc = j["accuracy"]
    assert acc["p_rel_l2_vs_oracle"] <= 1e-12 and acc["u_maxabs_vs_oracle"] <= 1e-12
    for mode in ("consistent_bands", "reference_bands"):
        rec = acc["vs_oracle"][mode]
        assert rec["p_rel_l2_vs_oracle"] <= 1e-12 and rec["u_maxabs_vs_oracle"] <= 1e-12, (mode, rec)
