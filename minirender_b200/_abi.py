"""ctypes mirror of include/minirender_b200.h and the loader of the CUDA library.

The structs here are byte-for-byte the C ABI the shared library exports. The library is the
in-tree ``minirender_b200/libminirender_b200.so`` built by ``minirender_b200.build``; loading
fails loudly when it is missing, there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(HERE, "libminirender_b200.so")

MR_OK = 0
STATUS_NAMES = {
    0: "MR_OK",
    1: "MR_INVALID_ARGUMENT",
    2: "MR_OUT_OF_RANGE",
    3: "MR_OVERFLOW",
    4: "MR_RUNTIME_ERROR",
    5: "MR_CANCELLED",
    6: "MR_LOGIC_ERROR",
    7: "MR_LENGTH_ERROR",
    8: "MR_CUDA_ERROR",
    9: "MR_OUT_OF_MEMORY",
    10: "MR_TIMEOUT",
}

DIFFUSE, CONDUCTOR, MIRROR, DIELECTRIC, CLOTH, SUBSURFACE = range(6)
MATERIAL_KINDS = {"diffuse": DIFFUSE, "conductor": CONDUCTOR, "mirror": MIRROR,
                  "dielectric": DIELECTRIC, "cloth": CLOTH, "subsurface": SUBSURFACE}
SAMPLING_BSDF, SAMPLING_LIGHT, SAMPLING_MIS = range(3)
SAMPLING_MODES = {"bsdf": SAMPLING_BSDF, "light": SAMPLING_LIGHT, "mis": SAMPLING_MIS}
RENDER_STATES = ["idle", "preparing", "running", "pausing", "paused", "finalizing",
                 "cancelling", "cancelled", "completed", "failed"]
JOB_STATES = ["queued", "running", "paused", "completed", "cancelled", "failed"]

f3 = C.c_float * 3
d3 = C.c_double * 3


class Camera(C.Structure):
    _fields_ = [("position", f3), ("target", f3), ("up", f3),
                ("vertical_fov_degrees", C.c_float), ("near_plane", C.c_float),
                ("far_plane", C.c_float), ("aperture_radius", C.c_float),
                ("focus_distance", C.c_float)]


class Material(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("base_color", f3), ("emission", f3),
                ("roughness", C.c_float), ("ior", C.c_float), ("double_sided", C.c_uint32),
                ("base_color_texture", C.c_uint32), ("texture_filter", C.c_uint32),
                ("normal_texture", C.c_uint32), ("normal_scale", C.c_float),
                ("normal_flip_y", C.c_uint32)]


class Texture(C.Structure):
    _fields_ = [("rgb", C.POINTER(C.c_float)), ("width", C.c_uint32), ("height", C.c_uint32)]


TEXTURE_FILTERS = {"nearest": 0, "bilinear": 1, "trilinear": 2}


class MeshCorner(C.Structure):
    _fields_ = [("position", C.c_uint32), ("normal", f3), ("uv", C.c_float * 2)]


class Mesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("position_count", C.c_uint32),
                ("corners", C.POINTER(MeshCorner)), ("triangle_count", C.c_uint32)]


class Instance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("material", C.c_uint32),
                ("object_to_world", C.c_float * 16), ("normal_to_world", C.c_float * 9)]


class DirectionalLight(C.Structure):
    _fields_ = [("direction", f3), ("color", f3), ("intensity", C.c_float)]


class MediumRegion(C.Structure):
    _fields_ = [("minimum", d3), ("maximum", d3), ("absorption", d3), ("scattering", d3),
                ("anisotropy", C.c_double), ("enabled", C.c_uint32)]


class SceneDesc(C.Structure):
    _fields_ = [("camera", Camera), ("environment", f3),
                ("meshes", C.POINTER(Mesh)), ("mesh_count", C.c_uint32),
                ("materials", C.POINTER(Material)), ("material_count", C.c_uint32),
                ("instances", C.POINTER(Instance)), ("instance_count", C.c_uint32),
                ("directional_lights", C.POINTER(DirectionalLight)),
                ("directional_light_count", C.c_uint32),
                ("media", C.POINTER(MediumRegion)), ("medium_count", C.c_uint32),
                ("textures", C.POINTER(Texture)), ("texture_count", C.c_uint32),
                ("environment_texture", C.c_uint32), ("environment_strength", C.c_float),
                ("environment_rotation_degrees", C.c_float)]


class BvhNode(C.Structure):
    _fields_ = [("minimum", f3), ("maximum", f3), ("first", C.c_uint32),
                ("right", C.c_uint32), ("count", C.c_uint32)]


class BvhDesc(C.Structure):
    _fields_ = [("nodes", C.POINTER(BvhNode)), ("node_count", C.c_uint32),
                ("order", C.POINTER(C.c_uint32)), ("primitive_count", C.c_uint32)]


class BuildSettings(C.Structure):
    _fields_ = [("split_references", C.c_uint32), ("split_factor", C.c_float),
                ("max_references", C.c_uint64), ("two_level", C.c_uint32)]


class IntegratorSettings(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("maximum_depth", C.c_uint32),
                ("russian_roulette", C.c_uint32), ("roulette_depth", C.c_uint32)]


class RenderSettings(C.Structure):
    _fields_ = [("width", C.c_uint64), ("height", C.c_uint64),
                ("samples_per_pixel", C.c_uint32), ("seed", C.c_uint64)]


class SessionSettings(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("tile_size", C.c_uint32),
                ("batch_samples", C.c_uint32)]


class TraceStatistics(C.Structure):
    _fields_ = [("bounds_tests", C.c_uint64), ("triangle_tests", C.c_uint64)]


class PathStatistics(C.Structure):
    _fields_ = [("geometry", TraceStatistics), ("paths", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("scattering_events", C.c_uint64),
                ("roulette_terminations", C.c_uint64),
                ("medium_scattering_events", C.c_uint64),
                ("subsurface_events", C.c_uint64), ("subsurface_distance", C.c_double)]

    def as_dict(self):
        return {"bounds_tests": self.geometry.bounds_tests,
                "triangle_tests": self.geometry.triangle_tests,
                "paths": self.paths, "shadow_rays": self.shadow_rays,
                "scattering_events": self.scattering_events,
                "roulette_terminations": self.roulette_terminations,
                "medium_scattering_events": self.medium_scattering_events}


class BvhStatistics(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("nodes", C.c_uint64), ("leaves", C.c_uint64),
                ("maximum_depth", C.c_uint64)]


class Ray(C.Structure):
    _fields_ = [("origin", f3), ("direction", f3), ("minimum", C.c_float),
                ("maximum", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("distance", C.c_float), ("instance_index", C.c_uint32),
                ("triangle_index", C.c_uint32), ("primitive", C.c_uint32),
                ("barycentric", f3), ("front_face", C.c_uint32)]


class RenderProgress(C.Structure):
    _fields_ = [("state", C.c_uint32), ("job_id", C.c_uint64),
                ("recorded_samples", C.c_uint64), ("total_samples", C.c_uint64),
                ("completed_pixels", C.c_uint64), ("worker_count", C.c_uint32),
                ("elapsed_seconds", C.c_double), ("statistics", PathStatistics),
                ("error", C.c_char * 256)]


class RenderPreview(C.Structure):
    _fields_ = [("job_id", C.c_uint64), ("revision", C.c_uint64),
                ("recorded_samples", C.c_uint64), ("width", C.c_uint64),
                ("height", C.c_uint64), ("available", C.c_uint32)]


P = C.POINTER
VP = C.c_void_p


class BatchSettings(C.Structure):
    _fields_ = [("wave_paths", C.c_uint64), ("trace_blocks_per_sm", C.c_uint32),
                ("shade_blocks_per_sm", C.c_uint32), ("sort_threshold", C.c_uint32),
                ("use_graphs", C.c_uint32), ("concurrent_waves", C.c_uint32)]


class BatchJob(C.Structure):
    _fields_ = [("scene", VP), ("integrator", IntegratorSettings), ("render", RenderSettings),
                ("rgb", P(C.c_float)), ("status", C.c_int)]


class BatchStatistics(C.Structure):
    _fields_ = [("waves", C.c_uint64), ("segments", C.c_uint64), ("samples", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("graph_launches", C.c_uint64),
                ("seconds", C.c_double), ("busy_seconds", C.c_double),
                ("device_seconds", C.c_double), ("paths", PathStatistics)]


class ServerSettings(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_jobs", C.c_uint32), ("policy", C.c_uint32),
                ("batch", BatchSettings)]


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_uint32), ("status", C.c_uint32), ("total_samples", C.c_uint64),
                ("completed_samples", C.c_uint64), ("submitted_seconds", C.c_double),
                ("admitted_seconds", C.c_double), ("finished_seconds", C.c_double),
                ("error", C.c_char * 256)]


class ServerStatistics(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "admitted", "completed", "cancelled", "failed",
                                          "waves", "segments", "samples", "kernel_launches",
                                          "graph_launches", "resident_bytes")] + \
               [("busy_seconds", C.c_double), ("elapsed_seconds", C.c_double)]


# Every exported symbol of include/minirender_b200.h with its ctypes signature.
SIGNATURES = {
    "mr_abi_version": (C.c_uint32, []),
    "mr_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "mr_scene_create": (C.c_int, [P(SceneDesc), P(BvhDesc), P(VP)]),
    "mr_scene_create_with": (C.c_int, [P(SceneDesc), P(BvhDesc), P(BuildSettings), P(VP)]),
    "mr_scene_destroy": (C.c_int, [VP]),
    "mr_scene_update_instances": (C.c_int, [VP, C.c_uint32, C.c_uint32, P(Instance)]),
    "mr_scene_update_mesh": (C.c_int, [VP, C.c_uint32, P(C.c_float), C.c_uint32]),
    "mr_scene_device_bytes": (C.c_int, [VP, P(C.c_uint64)]),
    "mr_scene_bvh_statistics": (C.c_int, [VP, P(BvhStatistics)]),
    "mr_scene_sah_cost": (C.c_int, [VP, P(C.c_double)]),
    "mr_scene_export_bvh": (C.c_int, [VP, P(BvhNode), C.c_uint32, P(C.c_uint32), C.c_uint32,
                                      P(C.c_uint32), P(C.c_uint32)]),
    "mr_scene_build_seconds": (C.c_int, [VP, P(C.c_double)]),
    "mr_intersect": (C.c_int, [VP, P(Ray), C.c_size_t, P(Hit), P(TraceStatistics)]),
    "mr_occluded": (C.c_int, [VP, P(Ray), C.c_size_t, P(C.c_uint8), P(TraceStatistics)]),
    "mr_trace_paths": (C.c_int, [VP, P(IntegratorSettings), P(Ray), P(C.c_uint64), C.c_size_t,
                                 P(C.c_float), P(PathStatistics)]),
    "mr_sample_pixels": (C.c_int, [VP, P(IntegratorSettings), P(RenderSettings),
                                   P(C.c_uint32), P(C.c_uint64), C.c_size_t, P(C.c_float),
                                   P(Ray), P(PathStatistics)]),
    "mr_capture_shadow_rays": (C.c_int, [VP, P(IntegratorSettings), P(RenderSettings),
                                         P(C.c_uint32), P(C.c_uint64), C.c_size_t, P(Ray),
                                         P(C.c_uint8), P(C.c_uint8)]),
    "mr_trace_paths_static": (C.c_int, [VP, P(IntegratorSettings), VP, VP, C.c_size_t, VP, VP]),
    "mr_render": (C.c_int, [VP, P(IntegratorSettings), P(RenderSettings), P(C.c_float),
                            P(PathStatistics)]),
    "mr_render_rows": (C.c_int, [VP, P(IntegratorSettings), P(RenderSettings), C.c_uint64,
                                 C.c_uint64, P(C.c_float), P(PathStatistics)]),
    "mr_render_device": (C.c_int, [VP, P(IntegratorSettings), P(RenderSettings), VP, VP,
                                   P(PathStatistics)]),
    "mr_display_image": (C.c_int, [P(C.c_float), C.c_uint64, C.c_uint64, C.c_double,
                                   P(C.c_float)]),
    "mr_set_kernel_timing": (C.c_int, [C.c_int]),
    "mr_kernel_timing": (C.c_int, [P(C.c_uint64), P(C.c_double), P(TraceStatistics),
                                   P(C.c_uint64)]),
    "mr_session_create": (C.c_int, [P(VP)]),
    "mr_session_destroy": (C.c_int, [VP]),
    "mr_session_start": (C.c_int, [VP, VP, P(RenderSettings), P(IntegratorSettings),
                                   P(SessionSettings)]),
    "mr_session_pause": (C.c_int, [VP, P(C.c_int)]),
    "mr_session_resume": (C.c_int, [VP, P(C.c_int)]),
    "mr_session_cancel": (C.c_int, [VP]),
    "mr_session_wait": (C.c_int, [VP]),
    "mr_session_wait_for": (C.c_int, [VP, C.c_uint32, P(C.c_int)]),
    "mr_session_progress": (C.c_int, [VP, P(RenderProgress)]),
    "mr_session_preview": (C.c_int, [VP, C.c_uint64, P(C.c_float), C.c_size_t,
                                     P(RenderPreview)]),
    "mr_render_batch": (C.c_int, [P(BatchJob), C.c_size_t, P(BatchSettings), P(BatchStatistics)]),
    "mr_batch_autotune": (C.c_int, [P(BatchJob), C.c_size_t, P(BatchSettings), P(C.c_double)]),
    "mr_server_create": (C.c_int, [P(ServerSettings), P(VP)]),
    "mr_server_destroy": (C.c_int, [VP]),
    "mr_server_submit": (C.c_int, [VP, VP, P(RenderSettings), P(IntegratorSettings), P(C.c_uint64)]),
    "mr_server_pause": (C.c_int, [VP, C.c_uint64, P(C.c_int)]),
    "mr_server_resume": (C.c_int, [VP, C.c_uint64, P(C.c_int)]),
    "mr_server_cancel": (C.c_int, [VP, C.c_uint64]),
    "mr_server_wait": (C.c_int, [VP, C.c_uint64, C.c_uint32, P(C.c_int)]),
    "mr_server_job_info": (C.c_int, [VP, C.c_uint64, P(JobInfo)]),
    "mr_server_result": (C.c_int, [VP, C.c_uint64, P(C.c_float), C.c_size_t]),
    "mr_server_preview": (C.c_int, [VP, C.c_uint64, P(C.c_float), C.c_size_t, P(C.c_uint64)]),
    "mr_server_release": (C.c_int, [VP, C.c_uint64]),
    "mr_server_get_statistics": (C.c_int, [VP, P(ServerStatistics)]),
    "mr_session_result": (C.c_int, [VP, P(C.c_float), C.c_size_t, P(C.c_uint64),
                                    P(C.c_uint64)]),
}


class MiniRenderError(RuntimeError):
    """A non-MR_OK status from the C ABI, carrying the status code and message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


_lock = threading.Lock()
_library = None


def load_library(path: str | None = None):
    """Loads libminirender_b200.so (raises if it has not been built)."""
    global _library
    with _lock:
        if _library is not None and path is None:
            return _library
        target = path or LIBRARY_PATH
        if not os.path.exists(target):
            raise ImportError(
                f"{target} is missing: build the CUDA library first "
                "(python -c 'import __graft_entry__ as g; g.build()')")
        lib = C.CDLL(target)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        if path is None:
            _library = lib
        return lib


def check(status: int, lib=None):
    if status != MR_OK:
        lib = lib or load_library()
        buffer = C.create_string_buffer(1024)
        lib.mr_last_error(buffer, 1024)
        raise MiniRenderError(status, buffer.value.decode(errors="replace"))
