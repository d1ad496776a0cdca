"""ctypes binding of the CPU oracle. TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this
module; the product (``minirender_b200``) never does. The oracle is the FP64 restatement of the
reference's offline path tracer in ``oracle/oracle.cpp``.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from minirender_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


def build():
    """Compiles oracle.cpp (make) into oracle/_build/."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _cpu_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " fma " in f.read()
    except OSError:
        return False


_lib = None


def lib():
    """The oracle library: liboracle.so (nofma without hardware FMA), or the variant the
    environment names in ORACLE_VARIANT ("contract": multiply-adds fused by the compiler;
    "f32offsets": ray offsets sized with float's epsilon, as on the FP32 device)."""
    global _lib
    if _lib is None:
        name = "liboracle.so" if _cpu_has_fma() else "liboracle_nofma.so"
        variant = os.environ.get("ORACLE_VARIANT")
        if variant == "contract":
            name = "liboracle_contract.so"
        elif variant == "f32offsets":
            name = "liboracle_f32offsets.so"
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        _declare(_lib)
    return _lib


class DRay(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("direction", C.c_double * 3),
                ("minimum", C.c_double), ("maximum", C.c_double)]


P = C.POINTER
VP = C.c_void_p
dp = P(C.c_double)


def _declare(l):
    sig = {
        "or_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
        "or_pcg_sequence": (None, [C.c_uint64, C.c_uint64, C.c_size_t, P(C.c_uint32)]),
        "or_stream_1d": (None, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_size_t, dp]),
        "or_sampler_state": (None, [C.c_uint64, C.c_uint64, C.c_uint64, P(C.c_uint64)]),
        "or_warp": (C.c_int, [C.c_int, dp, C.c_size_t, dp]),
        "or_distribution": (C.c_int, [dp, C.c_size_t, dp, C.c_size_t, dp, P(C.c_uint64), dp, dp]),
        "or_fresnel_dielectric": (C.c_int, [C.c_double, C.c_double, C.c_double, dp]),
        "or_bsdf_sample": (C.c_int, [P(_abi.Material), C.c_int, C.c_int, dp, C.c_double, dp, dp]),
        "or_bsdf_eval": (C.c_int, [P(_abi.Material), C.c_int, dp, dp, dp, dp, P(C.c_int)]),
        "or_power_heuristic": (C.c_int, [C.c_double, C.c_double, dp]),
        "or_phase": (C.c_int, [dp, dp, C.c_double, dp]),
        "or_sample_phase": (C.c_int, [dp, C.c_double, dp, dp]),
        "or_medium_distance": (C.c_int, [dp, dp, C.c_double, C.c_double, C.c_double, dp]),
        "or_scene_create": (C.c_int, [P(_abi.SceneDesc), P(_abi.BvhDesc),
                                      P(_abi.IntegratorSettings), P(VP)]),
        "or_scene_destroy": (None, [VP]),
        "or_bvh_counts": (C.c_int, [VP, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64),
                                    P(C.c_uint64)]),
        "or_bvh_export": (C.c_int, [VP, P(_abi.BvhNode), P(C.c_uint32)]),
        "or_sah_cost": (C.c_int, [VP, dp]),
        "or_primitives": (C.c_int, [VP, P(C.c_float)]),
        "or_intersect": (C.c_int, [VP, P(DRay), C.c_size_t, dp, P(C.c_uint64)]),
        "or_occluded": (C.c_int, [VP, P(DRay), C.c_size_t, P(C.c_uint8), P(C.c_uint64)]),
        "or_trace_paths": (C.c_int, [VP, P(DRay), P(C.c_uint64), C.c_size_t, dp,
                                     P(_abi.PathStatistics)]),
        "or_sample_pixels": (C.c_int, [VP, P(_abi.RenderSettings), P(C.c_uint32),
                                       P(C.c_uint64), C.c_size_t, dp, P(DRay),
                                       P(_abi.PathStatistics)]),
        "or_camera_rays": (C.c_int, [VP, dp, C.c_size_t, C.c_double, P(DRay)]),
        "or_render_rows": (C.c_int, [VP, P(_abi.RenderSettings), C.c_uint64, C.c_uint64,
                                     C.c_uint32, P(C.c_float), P(_abi.PathStatistics)]),
        "or_light_sample": (C.c_int, [VP, dp, C.c_double, dp, dp]),
        "or_light_table": (C.c_int, [VP, P(C.c_uint64), dp]),
        "or_display_image": (C.c_int, [P(C.c_float), C.c_uint64, C.c_uint64, C.c_double,
                                       P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(l, name)
        fn.restype = res
        fn.argtypes = args


class OracleError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _check(status):
    if status != 0:
        buf = C.create_string_buffer(1024)
        lib().or_last_error(buf, 1024)
        raise OracleError(status, buf.value.decode(errors="replace"))


def _ptr(a, ctype):
    return a.ctypes.data_as(P(ctype))


# ---- primitives ----

def pcg_sequence(seed, sequence, count):
    out = np.zeros(count, np.uint32)
    lib().or_pcg_sequence(seed, sequence, count, _ptr(out, C.c_uint32))
    return out


def stream_1d(seed, pixel, sample, count):
    out = np.zeros(count, np.float64)
    lib().or_stream_1d(seed, pixel, sample, count, _ptr(out, C.c_double))
    return out


def sampler_state(seed, pixel, sample):
    out = np.zeros(2, np.uint64)
    lib().or_sampler_state(seed, pixel, sample, _ptr(out, C.c_uint64))
    return int(out[0]), int(out[1])


WARPS = {"disk": 0, "sphere": 1, "hemisphere": 2, "cosine": 3, "triangle": 4}


def warp(kind, u):
    u = np.ascontiguousarray(u, np.float64).reshape(-1, 2)
    out = np.zeros((u.shape[0], 3), np.float64)
    _check(lib().or_warp(WARPS[kind], _ptr(u, C.c_double), u.shape[0], _ptr(out, C.c_double)))
    return out


def distribution(weights, us):
    w = np.ascontiguousarray(weights, np.float64)
    u = np.ascontiguousarray(us, np.float64)
    prob = np.zeros(len(w), np.float64)
    idx = np.zeros(len(u), np.uint64)
    mass = np.zeros(len(u), np.float64)
    remap = np.zeros(len(u), np.float64)
    _check(lib().or_distribution(_ptr(w, C.c_double), len(w), _ptr(u, C.c_double), len(u),
                                 _ptr(prob, C.c_double), _ptr(idx, C.c_uint64),
                                 _ptr(mass, C.c_double), _ptr(remap, C.c_double)))
    return prob, idx, mass, remap


def fresnel_dielectric(cosine, eta_i, eta_t):
    out = C.c_double()
    _check(lib().or_fresnel_dielectric(cosine, eta_i, eta_t, C.byref(out)))
    return out.value


def _material(kind, base_color=(1, 1, 1), roughness=0.5, ior=1.5):
    return _abi.Material(_abi.MATERIAL_KINDS[kind] if isinstance(kind, str) else kind,
                         _abi.f3(*base_color), _abi.f3(0, 0, 0), roughness, ior, 1)


def bsdf_sample(kind, wo, component, u, base_color=(1, 1, 1), roughness=0.5, ior=1.5,
                front_face=True, importance=False):
    m = _material(kind, base_color, roughness, ior)
    wo = np.ascontiguousarray(wo, np.float64)
    uu = np.ascontiguousarray(u, np.float64)
    out = np.zeros(11, np.float64)
    _check(lib().or_bsdf_sample(C.byref(m), int(front_face), int(importance),
                                _ptr(wo, C.c_double), component, _ptr(uu, C.c_double),
                                _ptr(out, C.c_double)))
    if out[10] == 0:
        return None
    return {"direction": out[0:3], "weight": out[3:6], "probability": out[6],
            "discrete": bool(out[7]), "event": int(out[8]), "eta": out[9]}


def bsdf_eval(kind, wo, wi, base_color=(1, 1, 1), roughness=0.5, ior=1.5, front_face=True):
    m = _material(kind, base_color, roughness, ior)
    wo = np.ascontiguousarray(wo, np.float64)
    wi = np.ascontiguousarray(wi, np.float64)
    value = np.zeros(3, np.float64)
    pdf = C.c_double()
    delta = C.c_int()
    _check(lib().or_bsdf_eval(C.byref(m), int(front_face), _ptr(wo, C.c_double),
                              _ptr(wi, C.c_double), _ptr(value, C.c_double), C.byref(pdf),
                              C.byref(delta)))
    return value, pdf.value, bool(delta.value)


def power_heuristic(a, b):
    out = C.c_double()
    _check(lib().or_power_heuristic(a, b, C.byref(out)))
    return out.value


def phase(wo, wi, g):
    wo = np.ascontiguousarray(wo, np.float64)
    wi = np.ascontiguousarray(wi, np.float64)
    out = C.c_double()
    _check(lib().or_phase(_ptr(wo, C.c_double), _ptr(wi, C.c_double), g, C.byref(out)))
    return out.value


def sample_phase(wo, g, u):
    wo = np.ascontiguousarray(wo, np.float64)
    uu = np.ascontiguousarray(u, np.float64)
    out = np.zeros(4, np.float64)
    _check(lib().or_sample_phase(_ptr(wo, C.c_double), g, _ptr(uu, C.c_double),
                                 _ptr(out, C.c_double)))
    return out[:3], out[3]


def medium_distance(absorption, scattering, length, channel_u, distance_u):
    a = np.ascontiguousarray(absorption, np.float64)
    s = np.ascontiguousarray(scattering, np.float64)
    out = np.zeros(5, np.float64)
    _check(lib().or_medium_distance(_ptr(a, C.c_double), _ptr(s, C.c_double), length,
                                    channel_u, distance_u, _ptr(out, C.c_double)))
    return bool(out[0]), out[1], out[2:5]


def display_image(linear, exposure=0.0):
    linear = np.ascontiguousarray(linear, np.float32)
    h, w = linear.shape[:2]
    out = np.zeros_like(linear)
    _check(lib().or_display_image(_ptr(linear, C.c_float), w, h, exposure,
                                  _ptr(out, C.c_float)))
    return out


def rays_to_d(origins, directions, minimum, maximum):
    n = len(origins)
    arr = (DRay * max(1, n))()
    o = np.asarray(origins, np.float64)
    d = np.asarray(directions, np.float64)
    mn = np.broadcast_to(np.asarray(minimum, np.float64), (n,))
    mx = np.broadcast_to(np.asarray(maximum, np.float64), (n,))
    buf = np.frombuffer(arr, dtype=np.float64).reshape(-1, 8)
    buf[:n, 0:3] = o
    buf[:n, 3:6] = d
    buf[:n, 6] = mn
    buf[:n, 7] = mx
    return arr


# ---- scene ----

def integrator(mode="mis", maximum_depth=8, russian_roulette=True, roulette_depth=3):
    return _abi.IntegratorSettings(_abi.SAMPLING_MODES[mode] if isinstance(mode, str) else mode,
                                   maximum_depth, int(russian_roulette), roulette_depth)


class OracleScene:
    """PathTracer + SceneBvh + LightSampler of the oracle over one snapshot."""

    def __init__(self, snapshot, settings=None, bvh=None):
        self.snapshot = snapshot
        self.settings = settings or integrator()
        handle = VP()
        bvh_ptr = C.pointer(bvh) if bvh is not None else None
        _check(lib().or_scene_create(snapshot.desc_pointer(), bvh_ptr,
                                     C.byref(self.settings), C.byref(handle)))
        self.handle = handle

    def __del__(self):
        if getattr(self, "handle", None):
            lib().or_scene_destroy(self.handle)
            self.handle = None

    def bvh_counts(self):
        n, p, leaves, depth = (C.c_uint64() for _ in range(4))
        _check(lib().or_bvh_counts(self.handle, C.byref(n), C.byref(p), C.byref(leaves),
                                   C.byref(depth)))
        return {"nodes": n.value, "triangles": p.value, "leaves": leaves.value,
                "maximum_depth": depth.value}

    def export_bvh(self):
        """Reference-layout BVH (nodes, order) and an mr_bvh_desc pointing into them."""
        c = self.bvh_counts()
        nodes = (_abi.BvhNode * max(1, c["nodes"]))()
        order = np.zeros(max(1, c["triangles"]), np.uint32)
        _check(lib().or_bvh_export(self.handle, nodes, _ptr(order, C.c_uint32)))
        desc = _abi.BvhDesc(nodes, c["nodes"], _ptr(order, C.c_uint32), c["triangles"])
        desc._keep = (nodes, order)
        return desc

    def sah_cost(self):
        out = C.c_double()
        _check(lib().or_sah_cost(self.handle, C.byref(out)))
        return out.value

    def primitives(self):
        n = self.bvh_counts()["triangles"]
        out = np.zeros((max(1, n), 3, 3), np.float32)
        _check(lib().or_primitives(self.handle, _ptr(out, C.c_float)))
        return out[:n]

    def intersect(self, origins, directions, minimum=1e-5, maximum=np.inf):
        rays = rays_to_d(origins, directions, minimum, maximum)
        n = len(origins)
        out = np.zeros((max(1, n), 18), np.float64)
        counters = np.zeros(2, np.uint64)
        _check(lib().or_intersect(self.handle, rays, n, _ptr(out, C.c_double),
                                  _ptr(counters, C.c_uint64)))
        return out[:n], counters

    def occluded(self, origins, directions, minimum=1e-5, maximum=np.inf):
        rays = rays_to_d(origins, directions, minimum, maximum)
        n = len(origins)
        out = np.zeros(max(1, n), np.uint8)
        counters = np.zeros(2, np.uint64)
        _check(lib().or_occluded(self.handle, rays, n, _ptr(out, C.c_uint8),
                                 _ptr(counters, C.c_uint64)))
        return out[:n].astype(bool), counters

    def trace_paths(self, origins, directions, minimum, maximum, keys):
        rays = rays_to_d(origins, directions, minimum, maximum)
        n = len(origins)
        keys = np.ascontiguousarray(keys, np.uint64).reshape(-1)
        out = np.zeros((max(1, n), 3), np.float64)
        stats = _abi.PathStatistics()
        _check(lib().or_trace_paths(self.handle, rays, _ptr(keys, C.c_uint64), n,
                                    _ptr(out, C.c_double), C.byref(stats)))
        return out[:n], stats.as_dict()

    def sample_pixels(self, render, pixels, samples, want_rays=False):
        pixels = np.ascontiguousarray(pixels, np.uint32).reshape(-1)
        samples = np.ascontiguousarray(samples, np.uint64)
        n = samples.shape[0]
        out = np.zeros((max(1, n), 3), np.float64)
        rays = (DRay * max(1, n))() if want_rays else None
        stats = _abi.PathStatistics()
        _check(lib().or_sample_pixels(self.handle, C.byref(render), _ptr(pixels, C.c_uint32),
                                      _ptr(samples, C.c_uint64), n, _ptr(out, C.c_double), rays,
                                      C.byref(stats)))
        if want_rays:
            r = np.frombuffer(rays, dtype=np.float64).reshape(-1, 8)[:n].copy()
            return out[:n], stats.as_dict(), r
        return out[:n], stats.as_dict()

    def camera_rays(self, uv, aspect):
        """Pinhole rays at film coordinates `uv` (n, 2) with the primary-ray diagnostic's clip
        interval: (n, 8) [origin, direction, minimum, maximum]."""
        uv = np.ascontiguousarray(uv, np.float64).reshape(-1, 2)
        n = len(uv)
        rays = (DRay * max(1, n))()
        _check(lib().or_camera_rays(self.handle, _ptr(uv, C.c_double), n, aspect, rays))
        return np.frombuffer(rays, dtype=np.float64).reshape(-1, 8)[:n].copy()

    def render(self, render, threads=None, rows=None, statistics=True):
        threads = threads or max(1, os.cpu_count() or 1)
        r0, r1 = rows if rows is not None else (0, render.height)
        out = np.zeros((r1 - r0, render.width, 3), np.float32)
        stats = _abi.PathStatistics()
        _check(lib().or_render_rows(self.handle, C.byref(render), r0, r1, threads,
                                    _ptr(out, C.c_float), C.byref(stats) if statistics else None))
        return out, stats.as_dict()

    def light_sample(self, reference, light_u, surface_u):
        ref = np.ascontiguousarray(reference, np.float64)
        su = np.ascontiguousarray(surface_u, np.float64)
        out = np.zeros(22, np.float64)
        _check(lib().or_light_sample(self.handle, _ptr(ref, C.c_double), light_u,
                                     _ptr(su, C.c_double), _ptr(out, C.c_double)))
        if out[0] == 0:
            return None
        return {"direction": out[1:4], "radiance": out[4:7], "distance": out[7],
                "probability": out[8], "discrete": bool(out[9]), "kind": int(out[10]),
                "emitter": int(out[11]), "position": out[12:15], "normal": out[15:18],
                "position_error": out[18:21]}

    def light_probabilities(self):
        n = C.c_uint64()
        _check(lib().or_light_table(self.handle, C.byref(n), None))
        out = np.zeros(max(1, n.value), np.float64)
        _check(lib().or_light_table(self.handle, C.byref(n), _ptr(out, C.c_double)))
        return out[:n.value]
