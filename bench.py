#!/usr/bin/env python
"""Throughput of the GPU offline path tracer on the uneven job mix, in Msamples/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 256 seeded render jobs. Each job is a Cornell room (5 walls, two boxes, a ceiling
light) filled with displaced icospheres up to its triangle count, drawn log-uniform in
[10k, 500k]; square images with pixel count log-uniform in [128^2, 1024^2]; samples per pixel
log-uniform in [4, 256]; maximum depth uniform in {4..12}; MIS, Russian roulette from depth 3.
One step renders all 256 jobs (about 3.2 G camera samples). Synthetic: the scenes and the job
table come from the package's seeded generators. Scenes are built with split references (the
result-neutral builder option for rooms around detailed objects).

Ours: the scenes are resident in HBM. `value` is the batched engine (mr_render_batch: jobs packed
into shared waves, CUDA graphs, concurrent wave lanes, shape from the autotuner run beforehand on
a calibration subset), camera samples of all ranks over the slowest rank's device time of K steps;
device time comes from CUDA events the engine records on its own streams around each step. The
inputs (scenes: tens of millions of triangles; path state: GBs) exceed L2, so no flush is added.
Beside it, on the same jobs and scenes: the plain one-job-per-call path (mr_render_device per job,
CUDA events on the caller's stream, kernel timing of the traversal kernel for the roofline), a
serving run (Poisson arrivals at 50 jobs/s through the render server, 5% cancelled, p50/p99
latency from submission to image in host memory; again at 16 jobs/s, a load one B200 keeps up
with), and the single 1M-triangle frame
(1920x1080, 64 spp, depth 12). `e2e` repeats the step through the public API from pinned host
memory: every step creates the 256 scenes (upload + GPU build, on 8 host threads) and renders
them with images read back to host memory. Multi-GPU runs are weak-scaled: each rank renders its own copy of the job
table with rank-specific render seeds; no collective on the data path.

Reference (--impl reference): the CPU oracle (the reference algorithm restated; the reference
itself does not build here) on the host cores, rank 0 only, each step a bounded band of rows of
four jobs spread over the table.
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
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Msamples/s"
JOBS = 256
TABLE_SEED = 3
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_BOUNDS_TEST = 24   # one FP32 AABB
BYTES_PER_TRIANGLE_TEST = 36  # one FP32 triangle
FLOPS_PER_BOUNDS_TEST = 24    # ~12 FP32 FMA-equivalents: six plane distances, min/max
FLOPS_PER_TRIANGLE_TEST = 80  # ~40 FP32 FMA-equivalents: shear, edge functions, error bound
SM_MAX_MHZ = 1965.0           # B200 maximum SM clock, when nvidia-smi reports none
CPU_SAMPLE_JOBS = (0, 64, 128, 192)
SERVE_RATE = 50.0             # jobs per second (the serving workload)
SUSTAINABLE_RATE = 16.0       # jobs per second that one B200 keeps up with on this job mix
CANCEL_FRACTION = 0.05


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-seconds", type=float, default=12.0,
                   help="target CPU time of the bounded CPU-baseline sample")
    p.add_argument("--serve-seconds", type=float, default=8.0,
                   help="length of the Poisson arrival window of the serving run")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--serve-rate", type=float, default=SERVE_RATE,
                   help="Poisson arrival rate of the serving run, jobs per second")
    p.add_argument("--leg", choices=["serve", "stress"], default=None,
                   help="run one secondary workload alone and print its JSON line")
    p.add_argument("--no-stress", dest="stress", action="store_false",
                   help="skip the 20M-triangle scene in a medium at 3840x2160, 256 spp, depth 16 "
                        "(about half a minute; rendered by default at N=1)")
    # Profiling aids (ncu captures); the defaults are the benchmark.
    p.add_argument("--jobs", type=int, default=JOBS, help="render only the first J jobs")
    p.add_argument("--no-autotune", action="store_true", help="default wave shape, no tuning")
    p.add_argument("--trace-sample", type=int, default=None, metavar="K",
                   help="render job K once on the plain path with kernel timing, print the "
                        "traversal work of its trace launches, and exit")
    return p.parse_args()


def trace_sample(k):
    """One plain render of job K with the traversal kernels' work counted: the algorithmic
    bytes an ncu capture of the same command divides its DRAM bytes by."""
    import torch
    from minirender_b200 import _abi, api
    job = job_table(JOBS)[k]
    scene = api.Scene(job_document(job).snapshot(), split_references=True)
    render = api.RenderSettings(job["width"], job["height"], job["samples_per_pixel"],
                                job["render_seed"])
    tracer = api.PathTracer(scene, api.IntegratorSettings("mis", job["maximum_depth"], True, 3))
    image = torch.empty(job["width"] * job["height"] * 3, dtype=torch.float32, device="cuda")
    lib = _abi.load_library()
    assert lib.mr_set_kernel_timing(1) == 0
    stats = tracer.render_device(render, image.data_ptr(), statistics=True)
    torch.cuda.synchronize()
    launches, seconds, all_launches = C.c_uint64(), C.c_double(), C.c_uint64()
    counted = _abi.TraceStatistics()
    lib.mr_kernel_timing(C.byref(launches), C.byref(seconds), C.byref(counted), C.byref(all_launches))
    lib.mr_set_kernel_timing(0)
    algorithmic = (BYTES_PER_BOUNDS_TEST * counted.bounds_tests +
                   BYTES_PER_TRIANGLE_TEST * counted.triangle_tests)
    kinds = ray_counts(stats)
    rays = sum(kinds.values())
    print(json.dumps({"job": k, **job, "trace_launches": launches.value,
                      "rays": rays, "rays_by_kind": kinds,
                      "rays_per_second": rays / seconds.value,
                      "bounds_tests": counted.bounds_tests,
                      "triangle_tests": counted.triangle_tests,
                      "algorithmic_bytes": algorithmic, "trace_seconds": seconds.value,
                      "all_launches": all_launches.value}), flush=True)
    return 0


def ray_counts(paths):
    """Rays traced, by kind, from path statistics: a camera ray per path, an extension ray per
    scattering event that survived roulette, and the shadow rays."""
    return {"primary": paths["paths"],
            "extension": paths["scattering_events"] - paths["roulette_terminations"],
            "shadow": paths["shadow_rays"]}


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def job_table(count):
    from minirender_b200 import scene as sc
    return sc.job_table(JOBS, TABLE_SEED)[:count]


def job_document(job):
    from minirender_b200 import scene as sc
    return sc.job_scene(job["triangles"], job["scene_seed"])


def config(table):
    """The workload, identical in both arms (the triangle total is what the job scenes build)."""
    from minirender_b200 import scene as sc
    return {"workload": f"uneven job mix: {len(table)} Cornell rooms with displaced icospheres, "
                        "10k-500k triangles, 128^2-1024^2 px, 4-256 spp, depth 4-12, mis",
            "jobs": len(table),
            "triangles_total": sum(sc.job_scene_triangles(j["triangles"]) for j in table),
            "samples_per_step": sum(j["width"] * j["height"] * j["samples_per_pixel"] for j in table),
            "job_table_seed": TABLE_SEED, "mode": "mis", "roulette_depth": 3,
            "l2": "no flush: scenes (tens of millions of triangles) and per-wave path state "
                  "(GBs) exceed the 126 MB L2"}


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


class CpuSample:
    """A bounded CPU-oracle sample of the workload: a central band of rows of four jobs spread
    over the table, each band sized for a share of a target CPU time."""

    def __init__(self, table, target_seconds):
        from minirender_b200 import _abi
        from oracle import pyoracle
        self.parts = []
        self.build = 0.0
        for k in CPU_SAMPLE_JOBS:
            if k >= len(table):
                continue
            job = table[k]
            t0 = time.perf_counter()
            o = pyoracle.OracleScene(job_document(job).snapshot(),
                                     pyoracle.integrator("mis", job["maximum_depth"], True, 3))
            self.build += time.perf_counter() - t0
            rs = _abi.RenderSettings(job["width"], job["height"], job["samples_per_pixel"],
                                     job["render_seed"])
            self.parts.append([o, rs, job, 1, k])
        per_job = target_seconds / max(1, len(self.parts))
        for part in self.parts:  # calibrate the band height per job
            rows, elapsed = 1, self._band(part, 1)
            while elapsed < 0.25 and rows < part[2]["height"]:
                rows = min(part[2]["height"], rows * 4)
                elapsed = self._band(part, rows)
            part[3] = int(max(1, min(part[2]["height"], round(per_job * rows / max(elapsed, 1e-6)))))

    @staticmethod
    def _band(part, rows):
        o, rs, job = part[0], part[1], part[2]
        r0 = job["height"] // 2 - rows // 2
        t0 = time.perf_counter()
        o.render(rs, threads=cpu_threads(), rows=(r0, r0 + rows), statistics=False)
        return time.perf_counter() - t0

    def run(self):
        seconds, samples = 0.0, 0
        for part in self.parts:
            seconds += self._band(part, part[3])
            samples += part[3] * part[2]["width"] * part[2]["samples_per_pixel"]
        return samples, seconds

    def describe(self, samples, seconds):
        bands = ", ".join(f"job {p[4]}: {p[3]} rows x {p[2]['width']} px x "
                          f"{p[2]['samples_per_pixel']} spp" for p in self.parts)
        return (f"central row bands ({bands}); {samples} samples in {seconds:.1f} s; oracle "
                f"BVH builds {self.build:.1f} s single-threaded (not in the rate); host has "
                f"{os.cpu_count()} hardware threads")


def cpu_baseline(table, target_seconds):
    sample = CpuSample(table, target_seconds)
    samples, seconds = sample.run()
    return {"value": samples / seconds / 1e6, "unit": METRIC, "cores": cpu_threads(),
            "kind": "port", "sample": sample.describe(samples, seconds)}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    table = job_table(args.jobs)
    # The same bounded sample as our arm's cpu_baseline (bands sized for --cpu-seconds), so the
    # two CPU figures of a run measure the same rows; each step renders it once.
    sample = CpuSample(table, args.cpu_seconds)
    for _ in range(args.warmup):
        sample.run()
    samples, seconds = 0, 0.0
    for _ in range(args.steps):
        n, s = sample.run()
        samples += n
        seconds += s
    value = samples / seconds / 1e6
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * seconds / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(table), "impl": "reference",
            "engine": "CPU oracle (the reference algorithm restated in FP64 C++), the reference's "
                      "serial SAH builder, tile-parallel render on the host threads",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cpu_threads(),
                             "kind": "port",
                             "sample": sample.describe(samples // max(1, args.steps),
                                                       seconds / max(1, args.steps))
                                       + " (per step)"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def serve(api, scenes, table, seconds, rng, rate=SERVE_RATE):
    """Poisson arrivals through the render server; returns latency and throughput figures."""
    server = api.RenderServer(policy="shortest_first", batch=api.BatchSettings())
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * seconds * 3) + 8))
    arrivals = arrivals[arrivals < seconds]
    picks = rng.integers(0, len(table), size=len(arrivals))
    # 5% of the jobs are cancelled at a uniform point of their expected life (their samples at
    # about the plain path's rate) after arrival.
    events = [(float(at), 0, i) for i, at in enumerate(arrivals)]
    for i, at in enumerate(arrivals):
        if rng.random() < CANCEL_FRACTION:
            job = table[picks[i]]
            life = job["width"] * job["height"] * job["samples_per_pixel"] / 250e6
            events.append((float(at + rng.uniform(0, max(life, 1e-3))), 1, i))
    events.sort()
    ids = {}
    t0 = time.perf_counter()
    for when, kind, i in events:
        delay = when - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        if kind == 0:
            job = table[picks[i]]
            render = api.RenderSettings(job["width"], job["height"], job["samples_per_pixel"],
                                        job["render_seed"])
            integrator = api.IntegratorSettings("mis", job["maximum_depth"], True, 3)
            ids[i] = server.submit(scenes[picks[i]], render, integrator)
        else:
            server.cancel(ids[i])
    latencies, samples, last, first = [], 0, 0.0, None
    states = {"completed": 0, "cancelled": 0, "failed": 0}
    for i in range(len(arrivals)):
        jid = ids[i]
        server.wait(jid)
        info = server.info(jid)
        states[info["state"]] = states.get(info["state"], 0) + 1
        if info["state"] == "completed":
            server.result(jid)  # the image in host memory, as a client receives it
            latencies.append(info["finished"] - info["submitted"])
            samples += info["total_samples"]
            last = max(last, info["finished"])
            first = info["submitted"] if first is None else min(first, info["submitted"])
        server.release(jid)
    stats = server.statistics()
    server.close()
    span = last - (first or 0.0)
    return {"arrival_rate_jobs_per_s": rate, "arrival_window_s": seconds,
            "jobs": len(arrivals), **states,
            "p50_latency_s": float(np.percentile(latencies, 50)) if latencies else None,
            "p99_latency_s": float(np.percentile(latencies, 99)) if latencies else None,
            "samples_per_s_M": samples / span / 1e6 if span > 0 else None,
            "waves": stats["waves"], "segments": stats["segments"],
            "latency": "submission to image in host memory (server clock)",
            "cancellation": "5% of jobs, at a uniform time within their expected duration "
                            "after arrival"}


def quintile_legs(api, jobs, tuned, plain):
    """Batched vs plain per fifth of the mix by samples per job (smallest first): where batching
    pays and where the plain path already fills the GPU."""
    order = sorted(range(len(jobs)), key=lambda k: jobs[k].render.width * jobs[k].render.height *
                   jobs[k].render.samples_per_pixel)
    out = []
    for q in range(5):
        part = [jobs[k] for k in order[q * len(jobs) // 5:(q + 1) * len(jobs) // 5]]
        if not part:
            continue
        counts = [j.render.width * j.render.height * j.render.samples_per_pixel for j in part]
        _, codes, info = api.render_batch(part, tuned, copy_images=False)
        assert all(c == 0 for c in codes), codes
        plain_s = plain(part)
        out.append({"jobs": len(part), "samples": sum(counts),
                    "samples_per_job": [min(counts), max(counts)],
                    "batched": sum(counts) / info["device_seconds"] / 1e6,
                    "plain": sum(counts) / plain_s / 1e6,
                    "batched_vs_plain": plain_s / info["device_seconds"], "unit": METRIC})
    return out


def quintile_bound(quintiles):
    """Upper bound on the mix's batched / plain ratio: every fifth of the mix rendered at the best
    rate any fifth reached batched (the GPU-saturated rate; batching cannot make a sample cheaper
    than a full GPU does) against the plain path's measured time."""
    if not quintiles:
        return None
    full = max(q["batched"] for q in quintiles)
    plain_s = sum(q["samples"] / q["plain"] for q in quintiles)
    ideal_s = sum(q["samples"] / full for q in quintiles)
    return {"value": plain_s / ideal_s, "full_gpu_rate": full, "unit": METRIC,
            "model": "plain seconds of every fifth / seconds at the best batched rate of any fifth"}


def preview_leg(api, jobs, tuned, plain):
    """Preview-sized renders of the same scenes (128x128, 4 spp, each job's depth): the regime in
    which one launch sequence per job leaves most of the GPU idle."""
    tiny = [api.BatchJob(j.scene, api.RenderSettings(128, 128, 4, j.render.seed), j.integrator)
            for j in jobs]
    tiny_samples = sum(j.render.width * j.render.height * j.render.samples_per_pixel for j in tiny)
    try:
        api.render_batch(tiny, tuned, copy_images=False)  # warm-up
        _, codes, info = api.render_batch(tiny, tuned, copy_images=False)
        assert all(c == 0 for c in codes), codes
        plain(tiny[:4])
        tiny_plain = plain(tiny)
        return {"jobs": len(tiny), "samples": tiny_samples, "render": "128x128, 4 spp",
                "batched": tiny_samples / info["device_seconds"] / 1e6,
                "plain": tiny_samples / tiny_plain / 1e6,
                "batched_vs_plain": tiny_plain / info["device_seconds"], "unit": METRIC}
    except Exception as error:  # a secondary leg: report it, keep the line
        return {"error": f"{type(error).__name__}: {error}"}


def timed_frames(tracer, render_settings, out, stream, count=1):
    """Device milliseconds of `count` frames after one warm-up frame (CUDA events on `stream`)."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tracer.render_device(render_settings[0], out.data_ptr(), stream.cuda_stream)
    e0.record(stream)
    for r in render_settings[:count]:
        tracer.render_device(r, out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


LARGE_BAND = (532, 548)


def large_frame_leg(api, sc, stream, with_cpu):
    """Config 2: the 1.02M-triangle frame, 1920x1080, 64 spp, depth 12, GPU-built tree (reference
    builder options); the CPU oracle renders a 16-row band of the same frame in the same run."""
    import torch
    snap = sc.large_scene().snapshot()
    large = api.Scene(snap)
    frame_render = api.RenderSettings(1920, 1080, 64, 1)
    frame_tracer = api.PathTracer(large, api.IntegratorSettings("mis", 12, True, 3))
    frame = torch.empty(1920 * 1080 * 3, dtype=torch.float32, device="cuda")
    frame_ms = timed_frames(frame_tracer, [frame_render], frame, stream)
    out = {"workload": "1920x1080 64 spp depth 12, 1.02M triangles (reference builder)",
           "ms": frame_ms, "value": 1920 * 1080 * 64 / frame_ms / 1e3, "unit": METRIC,
           "bvh_build_ms": 1e3 * large.build_seconds()}
    large.close()
    if with_cpu:
        from oracle import pyoracle
        o = pyoracle.OracleScene(snap, pyoracle.integrator("mis", 12, True, 3))
        t0 = time.perf_counter()
        o.render(frame_render.c(), threads=cpu_threads(), rows=LARGE_BAND, statistics=False)
        seconds = time.perf_counter() - t0
        band = (LARGE_BAND[1] - LARGE_BAND[0]) * 1920 * 64
        out["cpu_band"] = {"value": band / seconds / 1e6, "unit": METRIC, "cores": cpu_threads(),
                           "kind": "port", "rows": list(LARGE_BAND), "seconds": seconds,
                           "full_frame_seconds_extrapolated": seconds * 1080 / (LARGE_BAND[1] -
                                                                                LARGE_BAND[0]),
                           "sample": "rows 532-548 of the frame at full spp (the oracle's "
                                     "reference-builder tree; build not timed); the full "
                                     "frame's time extrapolated by row count"}
        out["gpu_vs_cpu"] = out["value"] / out["cpu_band"]["value"]
    return out


def large_frame_sharded(api, sc, rank, world):
    """Config 2 split into one row band per rank (mr_render_rows) and gathered on rank 0:
    the slowest rank's band time (host clock, after a barrier) plus the gather."""
    import torch
    import torch.distributed as dist
    from minirender_b200 import shard
    large = api.Scene(sc.large_scene().snapshot())
    tracer = api.PathTracer(large, api.IntegratorSettings("mis", 12, True, 3))
    render = api.RenderSettings(1920, 1080, 64, 1)
    shard.render_frame_sharded(tracer, render)  # warm-up
    dist.barrier()
    t0 = time.perf_counter()
    image = shard.render_frame_sharded(tracer, render)
    seconds = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    dist.all_reduce(seconds, op=dist.ReduceOp.MAX)
    large.close()
    ms = 1e3 * float(seconds.item())
    out = {"workload": "1920x1080 64 spp depth 12, 1.02M triangles, one row band per rank "
                       "gathered on rank 0", "ms": ms, "value": 1920 * 1080 * 64 / ms / 1e3,
           "unit": METRIC, "ranks": world}
    if rank == 0:
        out["image_mean"] = float(image.mean())
    return out


def config1_leg(api, sc, stream, with_cpu):
    """Config 1: the 36-triangle Cornell box at 512x512, 16 spp, depth 8, MIS, roulette from depth
    3, seeds 1-3, on the plain GPU path (device time), end to end through PathTracer.render (image
    in host memory), and the full frame of seed 1 on the CPU oracle in the same run."""
    import torch
    scene = api.Scene(sc.cornell_box().snapshot())
    settings = api.IntegratorSettings("mis", 8, True, 3)
    tracer = api.PathTracer(scene, settings)
    renders = [api.RenderSettings(512, 512, 16, seed) for seed in (1, 2, 3)]
    out_buf = torch.empty(512 * 512 * 3, dtype=torch.float32, device="cuda")
    samples = 512 * 512 * 16
    ms = timed_frames(tracer, renders, out_buf, stream, count=3)
    tracer.render(renders[0], statistics=False)
    t0 = time.perf_counter()
    for r in renders:
        tracer.render(r, statistics=False)
    e2e_seconds = time.perf_counter() - t0
    out = {"workload": "Cornell box, 36 triangles, 512x512, 16 spp, depth 8, mis, seeds 1-3",
           "ms_per_frame": ms / 3, "value": 3 * samples / ms / 1e3, "unit": METRIC,
           "e2e": {"value": 3 * samples / e2e_seconds / 1e6, "unit": METRIC,
                   "d2h_bytes_per_frame": 512 * 512 * 12,
                   "call": "mr_render (PathTracer::render) into host memory, per frame"}}
    scene.close()
    if with_cpu:
        from oracle import pyoracle
        o = pyoracle.OracleScene(sc.cornell_box().snapshot(), pyoracle.integrator("mis", 8, True, 3))
        t0 = time.perf_counter()
        o.render(renders[0].c(), threads=cpu_threads(), statistics=False)
        seconds = time.perf_counter() - t0
        out["cpu"] = {"value": samples / seconds / 1e6, "unit": METRIC, "cores": cpu_threads(),
                      "kind": "port", "seconds": seconds,
                      "sample": "the full 512x512x16 frame of seed 1"}
        out["e2e_vs_cpu"] = out["e2e"]["value"] / out["cpu"]["value"]
    return out


def stress_leg(api, sc, stream):
    """Config 5: 4,000 displaced icospheres (20.48M triangles) in one homogeneous medium,
    3840x2160, 256 spp, depth 16, after a 960x540x4 warm-up frame."""
    import torch
    doc = sc.stress_scene()
    t0 = time.perf_counter()
    big = api.Scene(doc.snapshot())
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    tracer = api.PathTracer(big, api.IntegratorSettings("mis", 16, True, 3))
    out = torch.empty(3840 * 2160 * 3, dtype=torch.float32, device="cuda")
    full = api.RenderSettings(3840, 2160, 256, 1)
    tracer.render_device(api.RenderSettings(960, 540, 4, 1), out.data_ptr(), stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    tracer.render_device(full, out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    result = {"workload": "4000 displaced icospheres (20.48M triangles) in one homogeneous "
                          "medium, 3840x2160, 256 spp, depth 16, reference builder",
              "ms": ms, "value": 3840 * 2160 * 256 / ms / 1e3, "unit": METRIC,
              "scene_create_s": build_s, "bvh_build_ms": 1e3 * big.build_seconds(),
              "triangles": doc.triangle_count}
    big.close()
    return result


def run_leg(args):
    """One secondary workload alone, for a recorded profile: `serve` (the Poisson request stream
    through the render server over --serve-seconds at --serve-rate jobs/s) or `stress`
    (config 5). Prints one JSON line with the clocks seen meanwhile."""
    import torch
    from minirender_b200 import api
    from minirender_b200 import scene as sc
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    clocks = ClockSampler(0)
    if args.leg == "serve":
        table = job_table(args.jobs)
        scenes = [api.Scene(job_document(j).snapshot(), split_references=True) for j in table]
        torch.cuda.synchronize()
        clocks.start()
        result = serve(api, scenes, table, args.serve_seconds, np.random.default_rng(50),
                       args.serve_rate)
    else:
        clocks.start()
        result = stress_leg(api, sc, stream)
    print(json.dumps({"leg": args.leg, "command": "python bench.py " + " ".join(sys.argv[1:]),
                      **result, "clocks": clocks.stop()}), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from minirender_b200 import _abi, api
    from minirender_b200 import scene as sc

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=5),
                                device_id=torch.device("cuda", local))
    lib = _abi.load_library()

    def barrier():
        if world > 1:
            dist.barrier()

    table = job_table(args.jobs)
    # One job table for the whole job. With N ranks it is partitioned by shard.partition_jobs
    # (longest processing time first on samples x depth) and every rank renders only its share:
    # strong scaling, no collective on the data path.
    mine = list(range(len(table)))
    if world > 1:
        from minirender_b200 import shard
        costs = [j["width"] * j["height"] * j["samples_per_pixel"] * (j["maximum_depth"] + 1)
                 for j in table]
        mine = shard.partition_jobs(costs, world)[rank]
    samples_total = sum(j["width"] * j["height"] * j["samples_per_pixel"] for j in table)
    t0 = time.perf_counter()
    snaps = [job_document(table[k]).snapshot() for k in mine]
    gen_seconds = time.perf_counter() - t0
    t0 = time.perf_counter()
    scenes = [api.Scene(s, split_references=True) for s in snaps]
    torch.cuda.synchronize()
    scene_seconds = time.perf_counter() - t0
    if world == 1:
        assert sum(s.triangle_count for s in snaps) == config(table)["triangles_total"]
    jobs = [api.BatchJob(s, api.RenderSettings(table[k]["width"], table[k]["height"],
                                               table[k]["samples_per_pixel"],
                                               table[k]["render_seed"]),
                         api.IntegratorSettings("mis", table[k]["maximum_depth"], True, 3))
            for s, k in zip(scenes, mine)]
    samples = sum(j.render.width * j.render.height * j.render.samples_per_pixel for j in jobs)

    # Autotuner on a calibration subset (every fourth job at a quarter of its samples: about a
    # sixteenth of the step, enough for the wave shapes to rank as they do on the whole), untimed.
    calib = [api.BatchJob(j.scene, api.RenderSettings(j.render.width, j.render.height,
                                                      max(1, j.render.samples_per_pixel // 4),
                                                      j.render.seed), j.integrator)
             for j in jobs[::4]]
    t0 = time.perf_counter()
    if args.no_autotune or not calib:
        tuned, tuned_rate = api.BatchSettings(), 0.0
    else:
        tuned, tuned_rate = api.autotune(calib)
    tune_seconds = time.perf_counter() - t0

    def step():
        if not jobs:  # a rank without a share (more ranks than jobs)
            return {"device_seconds": 0.0, "kernel_launches": 0, "waves": 0,
                    "paths": {"paths": 0, "scattering_events": 0, "roulette_terminations": 0,
                              "shadow_rays": 0}}
        _, codes, info = api.render_batch(jobs, tuned, copy_images=False)
        assert all(c == 0 for c in codes), codes
        return info

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    device_seconds, wall0 = 0.0, time.perf_counter()
    launches, waves = 0, 0
    rays = {"primary": 0, "extension": 0, "shadow": 0}
    for _ in range(args.steps):
        info = step()
        device_seconds += info["device_seconds"]
        launches += info["kernel_launches"]
        waves += info["waves"]
        for kind, n in ray_counts(info["paths"]).items():
            rays[kind] += n
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    barrier()
    clock_info = clocks.stop()
    worst = torch.tensor([device_seconds], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(worst, op=dist.ReduceOp.MAX)
    worst = float(worst.item())
    value = samples_total * args.steps / worst / 1e6
    own_batched_seconds = device_seconds / args.steps  # this rank's share, one step
    if world > 1:  # counters of the whole job
        totals = torch.tensor([launches, waves, *rays.values()], dtype=torch.float64,
                              device="cuda")
        dist.all_reduce(totals)
        launches, waves = int(totals[0].item()), int(totals[1].item())
        rays = {k: int(totals[2 + i].item()) for i, k in enumerate(rays)}

    # Plain path on the same jobs: one mr_render_device call per job.
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    image = torch.empty(max([j.render.width * j.render.height for j in jobs] or [1]) * 3,
                        dtype=torch.float32, device="cuda")

    def plain(part):
        """Device seconds of one mr_render_device call per job, on the caller's stream."""
        e0.record(stream)
        for j in part:
            api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                                stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    plain(jobs[:4])
    plain_seconds = plain(jobs)
    # The trace kernel's launch times for the roofline come from a second pass with per-launch
    # events; those make each wave wait for the host, so a frame's two lanes no longer overlap
    # and the pass is not the plain leg's time.
    assert lib.mr_set_kernel_timing(1) == 0
    plain(jobs)
    k_launches, ksec, all_launches = C.c_uint64(), C.c_double(), C.c_uint64()
    counted = _abi.TraceStatistics()
    lib.mr_kernel_timing(C.byref(k_launches), C.byref(ksec), C.byref(counted),
                         C.byref(all_launches))
    lib.mr_set_kernel_timing(0)
    plain_value = samples / max(plain_seconds, 1e-9) / 1e6

    quintiles = tiny_jobs = large_frame = config1 = None
    if world == 1:
        quintiles = quintile_legs(api, jobs, tuned, plain)
        tiny_jobs = preview_leg(api, jobs, tuned, plain)
        large_frame = large_frame_leg(api, sc, stream, not args.no_cpu_baseline)
        config1 = config1_leg(api, sc, stream, not args.no_cpu_baseline)
    else:
        large_frame = large_frame_sharded(api, sc, rank, world)

    # End to end through the public API from pinned host memory.
    e2e_value, h2d, d2h, e2e_phase = None, 0, 0, None
    if not args.no_e2e:
        h2d = sum(pin_snapshot(s) for s in snaps)
        d2h = sum(j.render.width * j.render.height * 3 * 4 for j in jobs)

        from concurrent.futures import ThreadPoolExecutor
        builders = ThreadPoolExecutor(8)

        phase = {"build": 0.0, "render": 0.0}

        def e2e_step():
            # Scenes are built on 8 host threads: construction runs on its own stream with
            # stream-ordered buffers, so builds overlap one another on the GPU. (Submitting each
            # job to the render server as its scene is ready was measured and is slower: the
            # builder's kernels wait behind the persistent render kernels.) With N ranks each
            # renders its share and rank 0 gathers every image (the one collective).
            t0 = time.perf_counter()
            fresh = list(builders.map(lambda s: api.Scene(s, split_references=True), snaps))
            t1 = time.perf_counter()
            batch = [api.BatchJob(f, j.render, j.integrator) for f, j in zip(fresh, jobs)]
            if batch:
                images, codes, _ = api.render_batch(batch, tuned)
                assert all(c == 0 for c in codes), codes
            else:
                images = []
            if world > 1:
                gathered = [None] * world if rank == 0 else None
                dist.gather_object(list(zip(mine, images)), gathered, dst=0)
                if rank == 0:
                    assert sum(len(g) for g in gathered) == len(table)
            phase["build"] += t1 - t0
            phase["render"] += time.perf_counter() - t1
            for f in fresh:
                f.close()

        e2e_step()
        barrier()
        torch.cuda.synchronize()
        phase = {"build": 0.0, "render": 0.0}
        w0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_seconds = torch.tensor([time.perf_counter() - w0], dtype=torch.float64, device="cuda")
        barrier()
        if world > 1:
            dist.all_reduce(e2e_seconds, op=dist.ReduceOp.MAX)
        e2e_value = samples_total * args.steps / float(e2e_seconds.item()) / 1e6
        e2e_phase = phase
        if world > 1:  # every rank's bytes: the job's totals
            counts = torch.tensor([h2d, d2h], dtype=torch.float64, device="cuda")
            dist.all_reduce(counts)
            h2d, d2h = int(counts[0].item()), int(counts[1].item())

    serving = sustainable = None
    if world == 1 and not args.no_serve:
        serving = serve(api, scenes, table, args.serve_seconds, np.random.default_rng(50))
        sustainable = serve(api, scenes, table, args.serve_seconds, np.random.default_rng(16),
                            SUSTAINABLE_RATE)

    stress = stress_leg(api, sc, stream) if args.stress and world == 1 else None

    peak, peak_kind = measured_peak()
    algorithmic = (BYTES_PER_BOUNDS_TEST * counted.bounds_tests +
                   BYTES_PER_TRIANGLE_TEST * counted.triangle_tests)
    achieved = algorithmic / ksec.value / 1e9 if ksec.value > 0 else 0.0
    per_launch = algorithmic / max(1, k_launches.value)
    # The arithmetic side of the same launches: FP32 operations (FMA-equivalents counted as two
    # flops) per test, against the nominal FP32 rate of the CUDA cores (128 lanes per SM).
    flops = FLOPS_PER_BOUNDS_TEST * counted.bounds_tests + FLOPS_PER_TRIANGLE_TEST * counted.triangle_tests
    props = torch.cuda.get_device_properties(local)
    max_mhz = (clock_info or {}).get("sm_max_mhz") or SM_MAX_MHZ
    fp32_peak = props.multi_processor_count * 128 * 2 * max_mhz * 1e6 / 1e12
    flops_achieved = flops / ksec.value / 1e12 if ksec.value > 0 else 0.0
    traffic, profile = None, {}
    tfile = os.path.join(ROOT, "profiles", "trace_kernel_traffic.txt")
    if os.path.exists(tfile):
        with open(tfile) as f:
            profile = json.load(f)
        ratio = profile.get("dram_bytes_per_algorithmic_byte")
        # DRAM bytes per algorithmic byte of the captured launches, applied to this run's
        # average launch.
        if ratio:
            traffic = ratio * per_launch
    avg_launch_s = ksec.value / max(1, k_launches.value)
    dram_gbs = traffic / avg_launch_s / 1e9 if traffic and avg_launch_s > 0 else None
    # What bounds the kernel: the algorithmic bytes are mostly served by L1/L2, so the DRAM side
    # runs far below the copy peak; the profile's issue and lane figures say why.
    limiter = ("issue and latency (divergent lanes), not DRAM: "
               f"{profile.get('lanes_active_per_instruction', '?')} of 32 lanes active per "
               f"instruction, issue active {profile.get('issue_active', '?')} of cycles "
               f"({profile.get('profile', 'profiles/trace_kernel_traffic.txt')})")

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": 1e3 * worst / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**config(table),
                       "engine": "batched: mr_render_batch, jobs packed into shared waves",
                       "bvh": "GPU binned SAH with split references",
                       "autotuned": {"wave_paths": tuned.wave_paths,
                                     "concurrent_waves": tuned.concurrent_waves,
                                     "sort_threshold": tuned.sort_threshold,
                                     "trace_blocks_per_sm": tuned.trace_blocks_per_sm,
                                     "calibration_Msamples_per_s": tuned_rate / 1e6,
                                     "tuning_s": tune_seconds},
                       "wall_ms_per_step": 1e3 * wall / args.steps,
                       "waves_per_step": waves / args.steps,
                       "rays": {"per_step": {kind: n // args.steps for kind, n in rays.items()},
                                "Grays_per_s": sum(rays.values()) / worst / 1e9,
                                "counted": "primary = camera paths, extension = scattering "
                                           "events that survived roulette, shadow = shadow "
                                           "rays (engine path statistics)"},
                       "scene_generation_s": gen_seconds, "scene_build_s": scene_seconds,
                       "plain_gpu": {"value": plain_value, "unit": METRIC,
                                     "ms_per_step": 1e3 * plain_seconds,
                                     "engine": "mr_render_device, one job per call"},
                       "batched_vs_plain": plain_seconds / max(own_batched_seconds, 1e-9),
                       "quintiles": quintiles,
                       "batched_vs_plain_bound": quintile_bound(quintiles),
                       "preview_jobs": tiny_jobs,
                       "config1": config1,
                       "serving": serving, "serving_sustainable": sustainable,
                       "large_frame": large_frame, "stress": stress},
            "roofline": {"bound": "hbm", "kernel": "trace_kernel (nearest-hit + shadow "
                                                   "traversal), plain leg of the same jobs",
                         "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": per_launch,
                         "launches": k_launches.value,
                         "avg_launch_ms": 1e3 * ksec.value / max(1, k_launches.value),
                         "bytes_model": "24 B per bounds test + 36 B per triangle test",
                         "dram": {"achieved": dram_gbs, "unit": "GB/s",
                                  "frac": dram_gbs / peak if dram_gbs else None,
                                  "from": "traffic per launch / average launch time"},
                         "limiter": limiter,
                         "fp32": {"achieved": flops_achieved, "peak": fp32_peak,
                                  "unit": "TFLOP/s", "frac": flops_achieved / fp32_peak,
                                  "peak_source": "nominal: SMs x 128 FP32 lanes x 2 x max SM clock",
                                  "flops_model": "24 per bounds test + 80 per triangle test"}},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "step": "256 scene uploads from pinned memory + GPU BVH builds (8 host "
                            "threads) + batched render + image read-back "
                            "(mr_scene_create_with + mr_render_batch)",
                    "scene_build_s_per_step": e2e_phase["build"] / args.steps if e2e_phase else None,
                    "render_s_per_step": e2e_phase["render"] / args.steps if e2e_phase else None},
            "gpu_launches": launches,
            "clocks": clock_info,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(table, args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.trace_sample is not None:
        return trace_sample(args.trace_sample)
    if args.impl == "reference":
        return run_reference(args)
    if args.leg:
        return run_leg(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
