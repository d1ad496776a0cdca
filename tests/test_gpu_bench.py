"""bench.py's own arm on the GPU prints one JSON line with the contract's keys: run on four jobs
of the mix with the default wave shape, one timed step, no serving, e2e, CPU or stress legs. The
secondary legs (per-quintile batched vs plain, config 1, the 1080p frame) report."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_prints_the_contract_line():
    result = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "3",
                             "--jobs", "4", "--no-autotune", "--no-serve", "--no-e2e",
                             "--no-cpu-baseline", "--no-stress"], cwd=ROOT, capture_output=True,
                            text=True,
                            timeout=900)
    assert result.returncode == 0, result.stderr[-4000:]
    line = json.loads(result.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "roofline", "e2e", "gpu_launches", "clocks"):
        assert key in line, key
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert "workload" in line["config"]
    roof = line["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in roof, key
    assert roof["achieved"] > 0 and 0 < roof["frac"] < 2
    assert 0 < roof["fp32"]["frac"] < 1
    assert line["gpu_launches"] > 0
    rays = line["config"]["rays"]["per_step"]
    samples = line["config"]["samples_per_step"]
    assert rays["primary"] == samples  # one camera ray per sample
    assert rays["extension"] > 0 and rays["shadow"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(line["clocks"])
    preview = line["config"]["preview_jobs"]
    assert "error" not in preview, preview
    assert preview["batched"] > 0 and preview["plain"] > 0
    assert all(q["batched_vs_plain"] > 0 for q in line["config"]["quintiles"])
    assert line["config"]["batched_vs_plain_bound"]["value"] > 0
    c1 = line["config"]["config1"]
    assert c1["value"] > 0 and c1["e2e"]["value"] > 0
    assert line["config"]["large_frame"]["value"] > 0
    assert line["roofline"]["dram"]["achieved"] is None or line["roofline"]["dram"]["achieved"] > 0
