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
    p.add_argument("--stress", action="store_true",
                   help="also render the 20M-triangle scene in a medium at 3840x2160, 256 spp, "
                        "depth 16 (about half a minute)")
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


def config(table, triangles):
    return {"workload": f"uneven job mix: {len(table)} Cornell rooms with displaced icospheres, "
                        "10k-500k triangles, 128^2-1024^2 px, 4-256 spp, depth 4-12, mis",
            "jobs": len(table), "triangles_total": triangles,
            "samples_per_step": sum(j["width"] * j["height"] * j["samples_per_pixel"] for j in table),
            "job_table_seed": TABLE_SEED, "mode": "mis", "roulette_depth": 3,
            "bvh": "GPU binned SAH with split references",
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
    budget = float(os.environ.get("BENCH_REFERENCE_SECONDS", 120.0))  # warmup + steps
    sample = CpuSample(table, budget / max(1, args.steps + args.warmup))
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
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(table, sum(j["triangles"] for j in table)), "impl": "reference",
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
    for job in table:  # weak scaling: every rank its own render seeds
        job["render_seed"] += 1000 * rank
    t0 = time.perf_counter()
    snaps = [job_document(j).snapshot() for j in table]
    gen_seconds = time.perf_counter() - t0
    t0 = time.perf_counter()
    scenes = [api.Scene(s, split_references=True) for s in snaps]
    torch.cuda.synchronize()
    scene_seconds = time.perf_counter() - t0
    triangles = sum(s.triangle_count for s in snaps)
    jobs = [api.BatchJob(s, api.RenderSettings(j["width"], j["height"], j["samples_per_pixel"],
                                               j["render_seed"]),
                         api.IntegratorSettings("mis", j["maximum_depth"], True, 3))
            for s, j in zip(scenes, table)]
    samples = sum(j.render.width * j.render.height * j.render.samples_per_pixel for j in jobs)

    # Autotuner on a calibration subset (every fourth job at 1/16 of its samples), untimed.
    calib = [api.BatchJob(j.scene, api.RenderSettings(j.render.width, j.render.height,
                                                      max(1, j.render.samples_per_pixel // 16),
                                                      j.render.seed), j.integrator)
             for j in jobs[::4]]
    t0 = time.perf_counter()
    if args.no_autotune:
        tuned, tuned_rate = api.BatchSettings(), 0.0
    else:
        tuned, tuned_rate = api.autotune(calib)
    tune_seconds = time.perf_counter() - t0

    def step():
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
    value = world * samples * args.steps / worst / 1e6

    # Plain path on the same jobs: one mr_render_device call per job.
    stream = torch.cuda.current_stream()
    image = torch.empty(max(j.render.width * j.render.height for j in jobs) * 3,
                        dtype=torch.float32, device="cuda")
    for j in jobs[:4]:
        api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                            stream.cuda_stream)
    torch.cuda.synchronize()
    assert lib.mr_set_kernel_timing(1) == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for j in jobs:
        api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                            stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_seconds = e0.elapsed_time(e1) / 1e3
    k_launches, ksec, all_launches = C.c_uint64(), C.c_double(), C.c_uint64()
    counted = _abi.TraceStatistics()
    lib.mr_kernel_timing(C.byref(k_launches), C.byref(ksec), C.byref(counted),
                         C.byref(all_launches))
    lib.mr_set_kernel_timing(0)
    plain_value = samples / plain_seconds / 1e6

    # The smaller half of the mix (by samples), batched and plain: the jobs batching is for.
    order = sorted(range(len(jobs)), key=lambda k: jobs[k].render.width * jobs[k].render.height *
                   jobs[k].render.samples_per_pixel)
    small = [jobs[k] for k in order[: len(jobs) // 2]]
    small_samples = sum(j.render.width * j.render.height * j.render.samples_per_pixel for j in small)
    api.render_batch(small, tuned, copy_images=False)  # warm-up
    _, _, info = api.render_batch(small, tuned, copy_images=False)
    small_batched = info["device_seconds"]
    e0.record(stream)
    for j in small:
        api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                            stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    small_plain = e0.elapsed_time(e1) / 1e3
    small_jobs = {"jobs": len(small), "samples": small_samples,
                  "batched": small_samples / small_batched / 1e6,
                  "plain": small_samples / small_plain / 1e6,
                  "batched_vs_plain": small_plain / small_batched, "unit": METRIC}

    # Preview-sized renders of the same scenes (128x128, 4 spp, each job's depth): the regime in
    # which one launch sequence per job leaves most of the GPU idle.
    tiny = [api.BatchJob(j.scene, api.RenderSettings(128, 128, 4, j.render.seed), j.integrator)
            for j in jobs]
    tiny_samples = sum(j.render.width * j.render.height * j.render.samples_per_pixel for j in tiny)
    try:
        api.render_batch(tiny, tuned, copy_images=False)  # warm-up
        _, codes, info = api.render_batch(tiny, tuned, copy_images=False)
        assert all(c == 0 for c in codes), codes
        tiny_batched = info["device_seconds"]
        for j in tiny[:4]:
            api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                                stream.cuda_stream)
        e0.record(stream)
        for j in tiny:
            api.PathTracer(j.scene, j.integrator).render_device(j.render, image.data_ptr(),
                                                                stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        tiny_plain = e0.elapsed_time(e1) / 1e3
        tiny_jobs = {"jobs": len(tiny), "samples": tiny_samples, "render": "128x128, 4 spp",
                     "batched": tiny_samples / tiny_batched / 1e6,
                     "plain": tiny_samples / tiny_plain / 1e6,
                     "batched_vs_plain": tiny_plain / tiny_batched, "unit": METRIC}
    except Exception as error:  # a secondary leg: report it, keep the line
        tiny_jobs = {"error": f"{type(error).__name__}: {error}"}

    # The single 1M-triangle frame (plain path), after one warm-up frame.
    large = api.Scene(sc.large_scene().snapshot())
    frame_render = api.RenderSettings(1920, 1080, 64, 1 + rank)
    frame_tracer = api.PathTracer(large, api.IntegratorSettings("mis", 12, True, 3))
    frame = torch.empty(1920 * 1080 * 3, dtype=torch.float32, device="cuda")
    frame_tracer.render_device(frame_render, frame.data_ptr(), stream.cuda_stream)
    e0.record(stream)
    frame_tracer.render_device(frame_render, frame.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    frame_ms = e0.elapsed_time(e1)
    large_frame = {"workload": "1920x1080 64 spp depth 12, 1.02M triangles (reference builder)",
                   "ms": frame_ms, "value": 1920 * 1080 * 64 / frame_ms / 1e3, "unit": METRIC,
                   "bvh_build_ms": 1e3 * large.build_seconds()}
    large.close()

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
            # stream-ordered buffers, so builds overlap one another on the GPU.
            t0 = time.perf_counter()
            fresh = list(builders.map(lambda s: api.Scene(s, split_references=True), snaps))
            t1 = time.perf_counter()
            batch = [api.BatchJob(f, j.render, j.integrator) for f, j in zip(fresh, jobs)]
            _, codes, _ = api.render_batch(batch, tuned)
            assert all(c == 0 for c in codes), codes
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
        e2e_value = world * samples * args.steps / float(e2e_seconds.item()) / 1e6
        e2e_phase = phase

    serving = sustainable = None
    if world == 1 and not args.no_serve:
        serving = serve(api, scenes, table, args.serve_seconds, np.random.default_rng(50))
        sustainable = serve(api, scenes, table, args.serve_seconds, np.random.default_rng(16),
                            SUSTAINABLE_RATE)

    stress = None
    if args.stress:
        doc = sc.stress_scene()
        t0 = time.perf_counter()
        big = api.Scene(doc.snapshot())
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0
        tracer = api.PathTracer(big, api.IntegratorSettings("mis", 16, True, 3))
        out = torch.empty(3840 * 2160 * 3, dtype=torch.float32, device="cuda")
        tracer.render_device(api.RenderSettings(960, 540, 4, 1), out.data_ptr(), stream.cuda_stream)
        full = api.RenderSettings(3840, 2160, 256, 1 + rank)
        e0.record(stream)
        tracer.render_device(full, out.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        stress = {"workload": "4000 displaced icospheres (20.48M triangles) in one homogeneous "
                              "medium, 3840x2160, 256 spp, depth 16, reference builder",
                  "ms": ms, "value": 3840 * 2160 * 256 / ms / 1e3, "unit": METRIC,
                  "scene_create_s": build_s, "bvh_build_ms": 1e3 * big.build_seconds()}
        big.close()

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
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "trace_kernel_traffic.txt")
    if os.path.exists(tfile):
        with open(tfile) as f:
            ratio = json.load(f).get("dram_bytes_per_algorithmic_byte")
        # DRAM bytes per algorithmic byte of the captured launches, applied to this run's
        # average launch.
        if ratio:
            traffic = ratio * per_launch

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": 1e3 * worst / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**config(table, triangles),
                       "engine": "batched: mr_render_batch, jobs packed into shared waves",
                       "autotuned": {"wave_paths": tuned.wave_paths,
                                     "concurrent_waves": tuned.concurrent_waves,
                                     "sort_threshold": tuned.sort_threshold,
                                     "trace_blocks_per_sm": tuned.trace_blocks_per_sm,
                                     "calibration_Msamples_per_s": tuned_rate / 1e6,
                                     "tuning_s": tune_seconds},
                       "wall_ms_per_step": 1e3 * wall / args.steps,
                       "waves_per_step": waves / args.steps,
                       "rays": {"per_step": {kind: n // args.steps for kind, n in rays.items()},
                                "Grays_per_s": world * sum(rays.values()) / worst / 1e9,
                                "counted": "primary = camera paths, extension = scattering "
                                           "events that survived roulette, shadow = shadow "
                                           "rays (engine path statistics)"},
                       "scene_generation_s": gen_seconds, "scene_build_s": scene_seconds,
                       "plain_gpu": {"value": plain_value, "unit": METRIC,
                                     "ms_per_step": 1e3 * plain_seconds,
                                     "engine": "mr_render_device, one job per call"},
                       "batched_vs_plain": value / plain_value,
                       "small_jobs": small_jobs,
                       "preview_jobs": tiny_jobs,
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
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
