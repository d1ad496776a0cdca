"""Host-side mirror of the reference's offline render interface over the C ABI.

``PathTracer`` and ``RenderSession`` keep the names, argument meaning and error behaviour of
MiniRender's classes (include/minirender/render/path_tracer.hpp:79-128,
include/minirender/render/render_session.hpp:82-115); every call goes through
``libminirender_b200.so`` and runs on the GPU. Errors raise ``MiniRenderError`` carrying the
C status that stands for the reference's exception type.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import MiniRenderError, check, load_library
from .scene import SceneDocument, Snapshot

__all__ = ["IntegratorSettings", "RenderSettings", "SessionSettings", "Scene", "PathTracer",
           "RenderSession", "MiniRenderError", "display_image", "BatchSettings", "BatchJob",
           "render_batch", "autotune", "RenderServer"]


@dataclass
class IntegratorSettings:
    """IntegratorSettings (include/minirender/render/path_tracer.hpp:21-35)."""

    mode: str = "mis"
    maximum_depth: int = 8
    russian_roulette: bool = True
    roulette_depth: int = 3

    def c(self) -> _abi.IntegratorSettings:
        return _abi.IntegratorSettings(_abi.SAMPLING_MODES[self.mode], self.maximum_depth,
                                       int(self.russian_roulette), self.roulette_depth)


@dataclass
class RenderSettings:
    """RenderSettings (include/minirender/render/path_tracer.hpp:38-49)."""

    width: int = 256
    height: int = 256
    samples_per_pixel: int = 64
    seed: int = 1

    def c(self) -> _abi.RenderSettings:
        return _abi.RenderSettings(self.width, self.height, self.samples_per_pixel, self.seed)


@dataclass
class SessionSettings:
    """SessionSettings (include/minirender/render/render_session.hpp:30-38)."""

    threads: int = 0
    tile_size: int = 16
    batch_samples: int = 4

    def c(self) -> _abi.SessionSettings:
        return _abi.SessionSettings(self.threads, self.tile_size, self.batch_samples)


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a if shape is None else a.reshape(shape)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def pack_rays(origins, directions, minimum, maximum) -> np.ndarray:
    """Packs rays into mr_ray records (8 float32 each)."""
    o = _f32(origins, (-1, 3))
    n = o.shape[0]
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3:6] = _f32(directions, (-1, 3))
    rays[:, 6] = np.broadcast_to(np.asarray(minimum, np.float32), (n,))
    rays[:, 7] = np.broadcast_to(np.asarray(maximum, np.float32), (n,))
    return rays


class Scene:
    """A snapshot uploaded to the current CUDA device with its BVH, lights and media
    (the construction half of PathTracer, src/render/path_tracer.cpp:111-120)."""

    def __init__(self, snapshot: Snapshot | SceneDocument, bvh: _abi.BvhDesc | None = None,
                 split_references: bool = False, split_factor: float = 0.0,
                 max_references: int = 0, two_level: bool = False):
        self.lib = load_library()
        if isinstance(snapshot, SceneDocument):
            snapshot = snapshot.snapshot()
        self.snapshot = snapshot
        handle = C.c_void_p()
        build = _abi.BuildSettings(int(split_references), split_factor, max_references,
                                   int(two_level))
        check(self.lib.mr_scene_create_with(snapshot.desc_pointer(),
                                            C.pointer(bvh) if bvh is not None else None,
                                            C.byref(build), C.byref(handle)), self.lib)
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mr_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        """Device memory the scene holds (geometry, trees, light and material tables)."""
        v = C.c_uint64()
        check(self.lib.mr_scene_device_bytes(self.handle, C.byref(v)), self.lib)
        return v.value

    def update_instances(self, first: int, document: SceneDocument):
        """Two-level scenes: takes the transforms of instances [first, first + k) from
        `document`'s objects first.. (same meshes and materials) and rebuilds the instance
        tree (mr_scene_update_instances)."""
        snap = document.snapshot()
        desc = snap.desc
        count = desc.instance_count - first
        base = C.addressof(desc.instances.contents) + first * C.sizeof(_abi.Instance)
        check(self.lib.mr_scene_update_instances(self.handle, first, count,
                                                 C.cast(base, C.POINTER(_abi.Instance))), self.lib)

    def update_mesh(self, mesh: int, positions):
        """Two-level scenes: new object-space positions (same count) of mesh `mesh`, whose tree is
        refit (mr_scene_update_mesh)."""
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        check(self.lib.mr_scene_update_mesh(self.handle, mesh, _ptr(p, C.c_float), p.shape[0]),
              self.lib)

    def statistics(self) -> dict:
        s = _abi.BvhStatistics()
        check(self.lib.mr_scene_bvh_statistics(self.handle, C.byref(s)), self.lib)
        return {"triangles": s.triangles, "nodes": s.nodes, "leaves": s.leaves,
                "maximum_depth": s.maximum_depth}

    def sah_cost(self) -> float:
        v = C.c_double()
        check(self.lib.mr_scene_sah_cost(self.handle, C.byref(v)), self.lib)
        return v.value

    def build_seconds(self) -> float:
        v = C.c_double()
        check(self.lib.mr_scene_build_seconds(self.handle, C.byref(v)), self.lib)
        return v.value

    def export_bvh(self):
        nodes_n, prims_n = C.c_uint32(), C.c_uint32()
        check(self.lib.mr_scene_export_bvh(self.handle, None, 0, None, 0, C.byref(nodes_n),
                                           C.byref(prims_n)), self.lib)
        nodes = (_abi.BvhNode * max(1, nodes_n.value))()
        order = np.zeros(max(1, prims_n.value), np.uint32)
        check(self.lib.mr_scene_export_bvh(self.handle, nodes, nodes_n.value,
                                           _ptr(order, C.c_uint32), prims_n.value, None, None),
              self.lib)
        return nodes, order[:prims_n.value], nodes_n.value

    # ---- SceneBvh queries (src/render/bvh.cpp:372-384) ----

    def intersect(self, origins, directions, minimum=1e-5, maximum=np.inf):
        rays = pack_rays(origins, directions, minimum, maximum)
        n = rays.shape[0]
        hits = (_abi.Hit * max(1, n))()
        stats = _abi.TraceStatistics()
        check(self.lib.mr_intersect(self.handle, C.cast(rays.ctypes.data, C.POINTER(_abi.Ray)), n,
                                    hits, C.byref(stats)), self.lib)
        raw = np.frombuffer(hits, dtype=np.dtype([("distance", "<f4"), ("instance", "<u4"),
                                                  ("triangle", "<u4"), ("primitive", "<u4"),
                                                  ("barycentric", "<f4", 3),
                                                  ("front_face", "<u4")]))[:n].copy()
        return raw, {"bounds_tests": stats.bounds_tests, "triangle_tests": stats.triangle_tests}

    def occluded(self, origins, directions, minimum=1e-5, maximum=np.inf):
        rays = pack_rays(origins, directions, minimum, maximum)
        n = rays.shape[0]
        out = np.zeros(max(1, n), np.uint8)
        stats = _abi.TraceStatistics()
        check(self.lib.mr_occluded(self.handle, C.cast(rays.ctypes.data, C.POINTER(_abi.Ray)), n,
                                   _ptr(out, C.c_uint8), C.byref(stats)), self.lib)
        return out[:n].astype(bool), {"bounds_tests": stats.bounds_tests,
                                      "triangle_tests": stats.triangle_tests}


class PathTracer:
    """PathTracer (include/minirender/render/path_tracer.hpp:79-128) on the GPU."""

    def __init__(self, scene: Scene | Snapshot | SceneDocument,
                 settings: IntegratorSettings | None = None, bvh=None):
        self.scene = scene if isinstance(scene, Scene) else Scene(scene, bvh)
        self.settings = settings or IntegratorSettings()
        self.lib = self.scene.lib
        # Validation happens in the library at every call (IntegratorSettings::validate).

    def trace(self, origins, directions, minimum, maximum, keys):
        """PathTracer::trace for many paths; keys[i] = (seed, pixel, sample) of the sampler."""
        rays = pack_rays(origins, directions, minimum, maximum)
        n = rays.shape[0]
        keys = np.ascontiguousarray(keys, np.uint64).reshape(-1)
        out = np.zeros((max(1, n), 3), np.float32)
        stats = _abi.PathStatistics()
        settings = self.settings.c()
        check(self.lib.mr_trace_paths(self.scene.handle, C.byref(settings),
                                      C.cast(rays.ctypes.data, C.POINTER(_abi.Ray)),
                                      _ptr(keys, C.c_uint64), n, _ptr(out, C.c_float),
                                      C.byref(stats)), self.lib)
        return out[:n], stats.as_dict()

    def sample_pixels(self, render: RenderSettings, pixels, samples, want_rays=False):
        """PathTracer::sample_pixel for many (x, y, sample) triples."""
        pixels = np.ascontiguousarray(pixels, np.uint32).reshape(-1)
        samples = np.ascontiguousarray(samples, np.uint64)
        n = samples.shape[0]
        out = np.zeros((max(1, n), 3), np.float32)
        rays = np.zeros((max(1, n), 8), np.float32) if want_rays else None
        stats = _abi.PathStatistics()
        settings, rs = self.settings.c(), render.c()
        check(self.lib.mr_sample_pixels(
            self.scene.handle, C.byref(settings), C.byref(rs), _ptr(pixels, C.c_uint32),
            _ptr(samples, C.c_uint64), n, _ptr(out, C.c_float),
            C.cast(rays.ctypes.data, C.POINTER(_abi.Ray)) if want_rays else None,
            C.byref(stats)), self.lib)
        if want_rays:
            return out[:n], stats.as_dict(), rays[:n]
        return out[:n], stats.as_dict()

    def capture_shadow_rays(self, render: RenderSettings, pixels, samples):
        """First shadow ray of each camera sample's path, whether one was traced, and its
        any-hit result (diagnostics for hit-record parity)."""
        pixels = np.ascontiguousarray(pixels, np.uint32).reshape(-1)
        samples = np.ascontiguousarray(samples, np.uint64)
        n = samples.shape[0]
        rays = np.zeros((max(1, n), 8), np.float32)
        has = np.zeros(max(1, n), np.uint8)
        occ = np.zeros(max(1, n), np.uint8)
        settings, rs = self.settings.c(), render.c()
        check(self.lib.mr_capture_shadow_rays(
            self.scene.handle, C.byref(settings), C.byref(rs), _ptr(pixels, C.c_uint32),
            _ptr(samples, C.c_uint64), n, C.cast(rays.ctypes.data, C.POINTER(_abi.Ray)),
            _ptr(has, C.c_uint8), _ptr(occ, C.c_uint8)), self.lib)
        return rays[:n], has[:n].astype(bool), occ[:n].astype(bool)

    def render(self, render: RenderSettings, statistics: bool = True):
        """PathTracer::render: (height, width, 3) float32 linear RGB, origin top-left."""
        out = np.zeros((render.height, render.width, 3), np.float32)
        stats = _abi.PathStatistics()
        settings, rs = self.settings.c(), render.c()
        check(self.lib.mr_render(self.scene.handle, C.byref(settings), C.byref(rs),
                                 _ptr(out, C.c_float), C.byref(stats) if statistics else None),
              self.lib)
        return out, stats.as_dict()

    def render_rows(self, render: RenderSettings, row_begin: int, row_end: int,
                    statistics: bool = False):
        """Rows [row_begin, row_end) of render(): ((row_end-row_begin), width, 3) float32, bit
        for bit the full image's rows."""
        out = np.zeros((max(0, row_end - row_begin), render.width, 3), np.float32)
        stats = _abi.PathStatistics()
        settings, rs = self.settings.c(), render.c()
        check(self.lib.mr_render_rows(self.scene.handle, C.byref(settings), C.byref(rs),
                                      row_begin, row_end,
                                      _ptr(out, C.c_float) if out.size else None,
                                      C.byref(stats) if statistics else None), self.lib)
        return (out, stats.as_dict()) if statistics else out

    def render_device(self, render: RenderSettings, device_ptr: int, stream: int = 0,
                      statistics: bool = False):
        """PathTracer::render into device memory (a pointer from the caller's allocator)."""
        stats = _abi.PathStatistics()
        settings, rs = self.settings.c(), render.c()
        check(self.lib.mr_render_device(self.scene.handle, C.byref(settings), C.byref(rs),
                                        C.c_void_p(device_ptr), C.c_void_p(stream),
                                        C.byref(stats) if statistics else None), self.lib)
        return stats.as_dict() if statistics else None


def display_image(linear: np.ndarray, exposure: float = 0.0) -> np.ndarray:
    """display_image (src/render/path_tracer.cpp:407-424)."""
    lib = load_library()
    linear = _f32(linear)
    h, w = linear.shape[:2]
    out = np.zeros_like(linear)
    check(lib.mr_display_image(_ptr(linear, C.c_float), w, h, exposure, _ptr(out, C.c_float)),
          lib)
    return out


class RenderSession:
    """RenderSession (include/minirender/render/render_session.hpp:82-115) on the GPU."""

    def __init__(self):
        self.lib = load_library()
        handle = C.c_void_p()
        check(self.lib.mr_session_create(C.byref(handle)), self.lib)
        self.handle = handle
        self._scene = None

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mr_session_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def start(self, scene: Scene, render: RenderSettings,
              integrator: IntegratorSettings | None = None,
              session: SessionSettings | None = None):
        integrator = integrator or IntegratorSettings()
        session = session or SessionSettings()
        rs, it, ss = render.c(), integrator.c(), session.c()
        check(self.lib.mr_session_start(self.handle, scene.handle, C.byref(rs), C.byref(it),
                                        C.byref(ss)), self.lib)
        self._scene = scene  # the scene must outlive the job
        self._render = render

    def pause(self) -> bool:
        ok = C.c_int()
        check(self.lib.mr_session_pause(self.handle, C.byref(ok)), self.lib)
        return bool(ok.value)

    def resume(self) -> bool:
        ok = C.c_int()
        check(self.lib.mr_session_resume(self.handle, C.byref(ok)), self.lib)
        return bool(ok.value)

    def cancel(self):
        check(self.lib.mr_session_cancel(self.handle), self.lib)

    def wait(self):
        check(self.lib.mr_session_wait(self.handle), self.lib)

    def wait_for(self, milliseconds: int) -> bool:
        done = C.c_int()
        check(self.lib.mr_session_wait_for(self.handle, milliseconds, C.byref(done)), self.lib)
        return bool(done.value)

    def progress(self) -> dict:
        p = _abi.RenderProgress()
        check(self.lib.mr_session_progress(self.handle, C.byref(p)), self.lib)
        return {"state": _abi.RENDER_STATES[p.state], "job_id": p.job_id,
                "recorded_samples": p.recorded_samples, "total_samples": p.total_samples,
                "completed_pixels": p.completed_pixels, "worker_count": p.worker_count,
                "elapsed_seconds": p.elapsed_seconds, "error": p.error.decode(errors="replace"),
                "statistics": p.statistics.as_dict()}

    def preview(self, maximum_dimension: int = 1024):
        info = _abi.RenderPreview()
        check(self.lib.mr_session_preview(self.handle, maximum_dimension, None, 0,
                                          C.byref(info)), self.lib)
        if not info.available:
            return None, info
        out = np.zeros((info.height, info.width, 3), np.float32)
        check(self.lib.mr_session_preview(self.handle, maximum_dimension, _ptr(out, C.c_float),
                                          out.size, C.byref(info)), self.lib)
        if not info.available:
            return None, info
        return out, info

    def result(self):
        w, h = C.c_uint64(), C.c_uint64()
        status = self.lib.mr_session_result(self.handle, None, 0, C.byref(w), C.byref(h))
        if status != _abi.MR_OK:
            return None
        out = np.zeros((h.value, w.value, 3), np.float32)
        check(self.lib.mr_session_result(self.handle, _ptr(out, C.c_float), out.size, None, None),
              self.lib)
        return out


@dataclass
class BatchSettings:
    """Wave shape of the multi-job engine (mr_batch_settings); zeros take the defaults."""

    wave_paths: int = 0
    trace_blocks_per_sm: int = 0
    shade_blocks_per_sm: int = 0
    sort_threshold: int = 0
    use_graphs: bool = True
    concurrent_waves: int = 0

    def c(self) -> _abi.BatchSettings:
        return _abi.BatchSettings(self.wave_paths, self.trace_blocks_per_sm,
                                  self.shade_blocks_per_sm, self.sort_threshold,
                                  int(self.use_graphs), self.concurrent_waves)

    @staticmethod
    def from_c(s: _abi.BatchSettings) -> "BatchSettings":
        return BatchSettings(s.wave_paths, s.trace_blocks_per_sm, s.shade_blocks_per_sm,
                             s.sort_threshold, bool(s.use_graphs), s.concurrent_waves)


@dataclass
class BatchJob:
    """One render of a batch: a scene, its integrator and render settings."""

    scene: Scene
    render: RenderSettings
    integrator: IntegratorSettings | None = None


def _batch_records(jobs, images):
    records = (_abi.BatchJob * max(1, len(jobs)))()
    for i, job in enumerate(jobs):
        records[i].scene = job.scene.handle
        records[i].integrator = (job.integrator or IntegratorSettings()).c()
        records[i].render = job.render.c()
        records[i].rgb = _ptr(images[i], C.c_float) if images is not None else None
    return records


def render_batch(jobs: list[BatchJob], settings: BatchSettings | None = None,
                 copy_images: bool = True):
    """Renders many jobs together (mr_render_batch). Returns the images ((H, W, 3) float32, None
    for a job that failed or when `copy_images` is false: the images then stay on the device
    and are dropped), the per-job status codes and the batch statistics."""
    lib = load_library()
    images = ([np.zeros((j.render.height, j.render.width, 3), np.float32) for j in jobs]
              if copy_images else None)
    records = _batch_records(jobs, images)
    stats = _abi.BatchStatistics()
    bs = (settings or BatchSettings()).c()
    status = lib.mr_render_batch(records, len(jobs), C.byref(bs), C.byref(stats))
    codes = [records[i].status for i in range(len(jobs))]
    if status != _abi.MR_OK and all(c == _abi.MR_OK for c in codes):
        check(status, lib)
    out = ([img if code == _abi.MR_OK else None for img, code in zip(images, codes)]
           if copy_images else [None] * len(jobs))
    info = {k: getattr(stats, k) for k in ("waves", "segments", "samples", "kernel_launches",
                                           "graph_launches", "seconds", "busy_seconds",
                                           "device_seconds")}
    info["paths"] = stats.paths.as_dict()
    return out, codes, info


def autotune(jobs: list[BatchJob]):
    """Runs the calibration jobs once per candidate wave shape, then the three fastest shapes
    (each also with fewer resident traversal blocks) twice more, and returns the best run's
    (BatchSettings, samples per device second)."""
    lib = load_library()
    records = _batch_records(jobs, None)
    best = _abi.BatchSettings()
    rate = C.c_double()
    check(lib.mr_batch_autotune(records, len(jobs), C.byref(best), C.byref(rate)), lib)
    return BatchSettings.from_c(best), rate.value


class RenderServer:
    """Request loop over the GPU (mr_server_*): admits jobs by HBM budget, keeps their
    accumulation buffers resident and renders every admitted job in shared waves."""

    POLICIES = {"shortest_first": 0, "arrival": 1}

    def __init__(self, hbm_budget_bytes: int = 0, max_jobs: int = 0, policy: str = "shortest_first",
                 batch: BatchSettings | None = None):
        self.lib = load_library()
        s = _abi.ServerSettings(hbm_budget_bytes, max_jobs, self.POLICIES[policy],
                                (batch or BatchSettings()).c())
        handle = C.c_void_p()
        check(self.lib.mr_server_create(C.byref(s), C.byref(handle)), self.lib)
        self.handle = handle
        self._sizes = {}
        self._scenes = {}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mr_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, scene: Scene, render: RenderSettings,
               integrator: IntegratorSettings | None = None) -> int:
        rs, it = render.c(), (integrator or IntegratorSettings()).c()
        job = C.c_uint64()
        check(self.lib.mr_server_submit(self.handle, scene.handle, C.byref(rs), C.byref(it),
                                        C.byref(job)), self.lib)
        self._sizes[job.value] = (render.height, render.width)
        self._scenes[job.value] = scene  # scenes must outlive their jobs
        return job.value

    def pause(self, job: int) -> bool:
        ok = C.c_int()
        check(self.lib.mr_server_pause(self.handle, job, C.byref(ok)), self.lib)
        return bool(ok.value)

    def resume(self, job: int) -> bool:
        ok = C.c_int()
        check(self.lib.mr_server_resume(self.handle, job, C.byref(ok)), self.lib)
        return bool(ok.value)

    def cancel(self, job: int):
        check(self.lib.mr_server_cancel(self.handle, job), self.lib)

    def wait(self, job: int, milliseconds: int = 0xFFFFFFFF) -> bool:
        done = C.c_int()
        check(self.lib.mr_server_wait(self.handle, job, milliseconds, C.byref(done)), self.lib)
        return bool(done.value)

    def info(self, job: int) -> dict:
        i = _abi.JobInfo()
        check(self.lib.mr_server_job_info(self.handle, job, C.byref(i)), self.lib)
        return {"state": _abi.JOB_STATES[i.state], "status": i.status,
                "total_samples": i.total_samples, "completed_samples": i.completed_samples,
                "submitted": i.submitted_seconds, "admitted": i.admitted_seconds,
                "finished": i.finished_seconds, "error": i.error.decode(errors="replace")}

    def result(self, job: int) -> np.ndarray:
        h, w = self._sizes[job]
        out = np.zeros((h, w, 3), np.float32)
        check(self.lib.mr_server_result(self.handle, job, _ptr(out, C.c_float), out.size), self.lib)
        return out

    def preview(self, job: int):
        h, w = self._sizes[job]
        out = np.zeros((h, w, 3), np.float32)
        n = C.c_uint64()
        check(self.lib.mr_server_preview(self.handle, job, _ptr(out, C.c_float), out.size,
                                         C.byref(n)), self.lib)
        return out, n.value

    def release(self, job: int):
        check(self.lib.mr_server_release(self.handle, job), self.lib)
        self._sizes.pop(job, None)
        self._scenes.pop(job, None)

    def statistics(self) -> dict:
        s = _abi.ServerStatistics()
        check(self.lib.mr_server_get_statistics(self.handle, C.byref(s)), self.lib)
        return {name: getattr(s, name) for name, _ in s._fields_}
