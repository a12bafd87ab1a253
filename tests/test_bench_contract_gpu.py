"""The benchmark's JSON line on the GPU: every key of the contract, with the
roofline, CPU baseline, end-to-end and clock records, for a short run of the
1 Mi-key workload."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_keeps_the_contract():
    from conftest import HAVE_GPU
    if not HAVE_GPU:
        pytest.skip("no GPU")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload",
                        "keys_u32_1M", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "e2e", "gpu_launches", "roofline", "cpu_baseline", "clocks"):
        assert key in line, key
    assert line["n_gpus"] == 1 and line["steps"] == 3 and line["warmup"] == 3
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["config"]["workload"] == "keys_u32_1M"
    assert line["gpu_launches"] > 0
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 4 * 1_048_576
    assert e2e["d2h_bytes_per_step"] == 4 * 1_048_576
    r = line["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["achieved"] > 0 and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    assert "traffic" in r
    cb = line["cpu_baseline"]
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] in ("port", "reference")
    assert cb["oracle_check"].startswith("GPU keys")
    assert "sm_mhz" in line["clocks"] and "reasons" in line["clocks"]
