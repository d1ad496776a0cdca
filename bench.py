#!/usr/bin/env python
"""Throughput of the GPU offline path tracer on the 1M-triangle workload, in Msamples/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the procedural ~1M-triangle scene (200 displaced 4-subdivision icospheres in a 20^3 box
on a ground quad, constant environment plus one directional light, thin lens with aperture 0.05
and focus distance 10), 1920x1080, 64 samples per pixel, maximum depth 12, MIS, Russian roulette
from depth 3. One step renders one full frame (132,710,400 camera samples). Synthetic, seeded.

Ours: the scene is resident in HBM (uploaded and BVH built once); `value` is samples of all ranks
over the slowest rank's device time for K frames (CUDA events on the launching stream, barrier +
synchronize on both sides, L2 flushed by a 256 MB write before every frame). `e2e` is the same
metric through the public API from pinned host buffers: every step creates the scene (upload +
GPU BVH build) and renders into a host image. Multi-GPU runs are weak-scaled: each rank renders
its own frame (seed = rank + 1), no collective on the data path.

Reference (--impl reference): the CPU oracle's tile-parallel render (the reference algorithm
restated; the reference itself does not build here) on the host cores, rank 0 only, each step a
bounded band of rows of the same frame.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WIDTH, HEIGHT, SPP, DEPTH = 1920, 1080, 64, 12
METRIC = "Msamples/s"
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_BOUNDS_TEST = 24   # one FP32 AABB
BYTES_PER_TRIANGLE_TEST = 36  # one FP32 triangle


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-seconds", type=float, default=12.0,
                   help="target CPU time of the bounded CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    # Profiling aids (ncu captures of a smaller frame); the defaults are the benchmark.
    p.add_argument("--resolution", default=None, help="WxH override, e.g. 960x540")
    p.add_argument("--spp", type=int, default=None)
    p.add_argument("--no-e2e", action="store_true")
    args = p.parse_args()
    global WIDTH, HEIGHT, SPP
    if args.resolution:
        WIDTH, HEIGHT = (int(v) for v in args.resolution.lower().split("x"))
    if args.spp:
        SPP = args.spp
    return args


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def workload():
    from minirender_b200 import scene as sc
    return sc.large_scene()


def config(triangles):
    return {"workload": "procedural-1M-triangles 1920x1080 64spp depth12 mis",
            "triangles": triangles, "width": WIDTH, "height": HEIGHT, "spp": SPP,
            "maximum_depth": DEPTH, "mode": "mis", "roulette_depth": 3,
            "samples_per_frame": WIDTH * HEIGHT * SPP,
            "l2": "256 MB write before every timed frame (included); per-frame path state "
                  "~1.8 GB > L2"}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        rows = [line.strip().split(", ") for line in self.file if line.strip()]
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9
                          for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def pin_snapshot(snapshot):
    """Moves every mesh buffer of the snapshot into pinned host memory (torch) and repoints the
    descriptor; returns the host->device byte count of one scene upload."""
    import torch
    desc = snapshot.desc
    keep = []
    total = 0
    for i in range(desc.mesh_count):
        m = desc.meshes[i]
        pos = np.ctypeslib.as_array(m.positions, shape=(3 * m.position_count,))
        cor_bytes = 24 * 3 * m.triangle_count
        cor = np.ctypeslib.as_array(C.cast(m.corners, C.POINTER(C.c_uint8)), shape=(cor_bytes,))
        p = torch.empty(pos.size, dtype=torch.float32, pin_memory=True)
        c = torch.empty(cor_bytes, dtype=torch.uint8, pin_memory=True)
        p.numpy()[:] = pos
        c.numpy()[:] = cor
        desc.meshes[i].positions = C.cast(p.data_ptr(), C.POINTER(C.c_float))
        desc.meshes[i].corners = C.cast(c.data_ptr(), type(m.corners))
        keep += [p, c]
        total += pos.nbytes + cor_bytes
    total += desc.instance_count * 108 + desc.material_count * 40
    snapshot._keep.append(keep)
    return total


def cpu_threads():
    """RenderSession's automatic worker count: hardware threads - 1, at most 32
    (src/render/render_session.cpp:386-392)."""
    hw = os.cpu_count() or 1
    return max(1, min(hw - 1 if hw > 1 else 1, 32))


def cpu_render_band(oracle_scene, rows, seed=1):
    from minirender_b200 import _abi
    rs = _abi.RenderSettings(WIDTH, HEIGHT, SPP, seed)
    r0 = HEIGHT // 2 - rows // 2
    t0 = time.perf_counter()
    oracle_scene.render(rs, threads=cpu_threads(), rows=(r0, r0 + rows), statistics=False)
    return time.perf_counter() - t0


def calibrated_rows(oracle_scene, target_seconds):
    rows, elapsed = 1, cpu_render_band(oracle_scene, 1)
    while elapsed < 0.5 and rows < HEIGHT:
        rows = min(HEIGHT, rows * 4)
        elapsed = cpu_render_band(oracle_scene, rows)
    per_row = elapsed / rows
    return int(max(1, min(HEIGHT, round(target_seconds / per_row))))


def cpu_baseline(snapshot, target_seconds):
    from oracle import pyoracle
    t0 = time.perf_counter()
    o = pyoracle.OracleScene(snapshot, pyoracle.integrator("mis", DEPTH, True, 3))
    build = time.perf_counter() - t0
    rows = calibrated_rows(o, target_seconds)
    seconds = cpu_render_band(o, rows)
    samples = rows * WIDTH * SPP
    return {"value": samples / seconds / 1e6, "unit": METRIC, "cores": cpu_threads(),
            "kind": "port",
            "sample": f"{rows} rows x 1920 px x 64 spp ({samples} samples) of the same frame, "
                      f"central band, {seconds:.1f} s; BVH build {build:.2f} s single-threaded "
                      f"(not in the rate); host has {os.cpu_count()} hardware threads"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    from oracle import pyoracle
    doc = workload()
    snap = doc.snapshot()
    o = pyoracle.OracleScene(snap, pyoracle.integrator("mis", DEPTH, True, 3))
    total_budget = float(os.environ.get("BENCH_REFERENCE_SECONDS", 120.0))  # warmup + steps
    rows = calibrated_rows(o, total_budget / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_render_band(o, rows)
    seconds = sum(cpu_render_band(o, rows) for _ in range(args.steps))
    samples = rows * WIDTH * SPP * args.steps
    value = samples / seconds / 1e6
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * seconds / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(snap.triangle_count), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cpu_threads(),
                             "kind": "port",
                             "sample": f"{rows} central rows x 1920 px x 64 spp per step"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from minirender_b200 import _abi, api

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=5),
                                device_id=torch.device("cuda", local))
    lib = _abi.load_library()

    doc = workload()
    snap = doc.snapshot()
    seed = rank + 1
    render = api.RenderSettings(WIDTH, HEIGHT, SPP, seed)
    integrator = api.IntegratorSettings("mis", DEPTH, True, 3)
    scene = api.Scene(snap)
    tracer = api.PathTracer(scene, integrator)
    stream = torch.cuda.current_stream()
    image = torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def frame():
        flush.fill_(1)
        tracer.render_device(render, image.data_ptr(), stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        frame()
    torch.cuda.synchronize()

    check = lib.mr_set_kernel_timing(1)
    assert check == 0
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        frame()
    stop.record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    seconds = start.elapsed_time(stop) / 1e3
    launches, ksec, all_launches = C.c_uint64(), C.c_double(), C.c_uint64()
    counted = _abi.TraceStatistics()
    lib.mr_kernel_timing(C.byref(launches), C.byref(ksec), C.byref(counted), C.byref(all_launches))
    lib.mr_set_kernel_timing(0)
    worst = torch.tensor([seconds], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(worst, op=dist.ReduceOp.MAX)
    worst = float(worst.item())
    samples = WIDTH * HEIGHT * SPP
    value = world * samples * args.steps / worst / 1e6

    # Path statistics of one frame (outside the timed region).
    stats = tracer.render_device(render, image.data_ptr(), stream.cuda_stream, statistics=True)
    torch.cuda.synchronize()

    # End to end through the public API from pinned host memory.
    if args.no_e2e:
        e2e_value, h2d, d2h = None, 0, 0
        args_e2e = False
    else:
        args_e2e = True
    h2d = pin_snapshot(snap) if args_e2e else 0
    d2h = WIDTH * HEIGHT * 3 * 4 if args_e2e else 0

    def e2e_step():
        s = api.Scene(snap)
        out, _ = api.PathTracer(s, integrator).render(render, statistics=False)
        s.close()
        return out

    e2e_value = None
    if args_e2e:
        e2e_step()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_seconds = torch.tensor([e0.elapsed_time(e1) / 1e3], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(e2e_seconds, op=dist.ReduceOp.MAX)
        e2e_value = world * samples * args.steps / float(e2e_seconds.item()) / 1e6

    peak, peak_kind = measured_peak()
    algorithmic = (BYTES_PER_BOUNDS_TEST * counted.bounds_tests +
                   BYTES_PER_TRIANGLE_TEST * counted.triangle_tests)
    achieved = algorithmic / ksec.value / 1e9 if ksec.value > 0 else 0.0
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "extend_kernel_traffic.txt")
    if os.path.exists(tfile):
        with open(tfile) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": 1e3 * worst / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**config(snap.triangle_count),
                       "bvh_build_ms": 1e3 * scene.build_seconds(),
                       "rays_per_frame": {"camera": stats["paths"],
                                          "extension": stats["scattering_events"],
                                          "shadow": stats["shadow_rays"]},
                       "bounds_tests_per_frame": stats["bounds_tests"],
                       "triangle_tests_per_frame": stats["triangle_tests"]},
            "roofline": {"bound": "hbm", "kernel": "extend_kernel (nearest-hit traversal)",
                         "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": algorithmic / max(1, launches.value),
                         "launches": launches.value,
                         "avg_launch_ms": 1e3 * ksec.value / max(1, launches.value),
                         "bytes_model": "24 B per bounds test + 36 B per triangle test"},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "step": "scene upload from pinned memory + GPU BVH build + render + "
                            "image read-back (mr_scene_create + mr_render)"},
            "gpu_launches": all_launches.value,
            "clocks": clock_info,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(snap, args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
