"""bench.py on the CPU: the reference arm (the CPU oracle on the host cores) prints one JSON line
with the contract's keys, run on a small budget here; the batched/plain bound the GPU arm reports
is the plain path's time over the time at the best batched rate of any fifth of the mix."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    result = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                             "--warmup", "1", "--jobs", "8", "--cpu-seconds", "1"], cwd=ROOT,
                            capture_output=True, text=True, timeout=600)
    assert result.returncode == 0, result.stderr
    line = json.loads(result.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert "workload" in line["config"]
    # The workload description is the one the GPU arm prints: the job scenes' exact triangles.
    sys.path.insert(0, ROOT)
    import bench
    from minirender_b200 import scene as sc
    table = sc.job_table(256, bench.TABLE_SEED)[:8]
    assert line["config"] == bench.config(table)
    assert line["config"]["triangles_total"] == sum(
        sc.job_scene_triangles(j["triangles"]) for j in table)


def test_quintile_bound_is_plain_time_over_time_at_the_best_batched_rate():
    sys.path.insert(0, ROOT)
    import bench
    # Two fifths: 100 M samples at 200 plain / 300 batched, 900 M samples at 400 / 390.
    quintiles = [{"samples": 100e6, "plain": 200.0, "batched": 300.0},
                 {"samples": 900e6, "plain": 400.0, "batched": 390.0}]
    bound = bench.quintile_bound(quintiles)
    plain_s = 100e6 / 200.0 + 900e6 / 400.0
    ideal_s = 1000e6 / 390.0
    assert abs(bound["value"] - plain_s / ideal_s) < 1e-12 and bound["full_gpu_rate"] == 390.0
    # A mix whose batched rates never beat the plain ones is bounded by the best of them.
    flat = [{"samples": 1e6, "plain": 100.0, "batched": 100.0}] * 5
    assert abs(bench.quintile_bound(flat)["value"] - 1.0) < 1e-12
    assert bench.quintile_bound([]) is None
