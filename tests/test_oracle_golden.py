"""Pins the CPU oracle to the reference's own golden vectors and known-answer tests.

Every test restates one case of the reference's Catch2 suite (file:line in the MiniRender tree)
against oracle/oracle.cpp. These run without a GPU.
"""

import math

import numpy as np
import pytest

from minirender_b200 import _abi
from minirender_b200.scene import (Camera, DirectionalLight, Material, MeshData, SceneDocument,
                                   SceneObject, Transform, box_mesh, quad_mesh)

PI = math.pi


def check_frequency(count, probability, total):
    """5 standard errors + 8 (tests/sampling_tests.cpp:51-55)."""
    expected = probability * total
    tolerance = 5 * math.sqrt(expected * (1 - probability)) + 8
    assert abs(count - expected) < tolerance


# ---- sampling (tests/sampling_tests.cpp) ----

def test_pcg_reference_sequence(oracle):
    # tests/sampling_tests.cpp:58-63
    assert oracle.pcg_sequence(42, 54, 6).tolist() == [
        0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]


def test_sample_streams_are_keyed_by_seed_pixel_sample(oracle):
    # tests/sampling_tests.cpp:64-82
    a = oracle.stream_1d(12, 0, 7, 32)
    assert np.array_equal(a, oracle.stream_1d(12, 0, 7, 32))
    assert not np.array_equal(a, oracle.stream_1d(12, 1, 7, 32))
    assert oracle.stream_1d(12, 0, 7, 1)[0] != oracle.stream_1d(12, 0, 8, 1)[0]
    assert oracle.stream_1d(12, 0, 7, 1)[0] != oracle.stream_1d(13, 0, 7, 1)[0]
    assert np.all((a >= 0) & (a < 1))


def test_warps_match_analytic_moments(oracle):
    # tests/sampling_tests.cpp:84-138
    count = 100000
    u = oracle.stream_1d(914, 21, 0, 2 * count).reshape(-1, 2)
    disk = oracle.warp("disk", u)[:, :2]
    r2 = (disk ** 2).sum(1)
    assert r2.max() <= 1 + 1e-12
    assert abs(r2.mean() - 0.5) < 0.006
    sphere = oracle.warp("sphere", u)
    assert np.allclose(np.linalg.norm(sphere, axis=1), 1, atol=1e-12)
    assert np.linalg.norm(sphere.mean(0)) < 0.01
    cosine = oracle.warp("cosine", u)
    assert cosine[:, 2].min() >= 0
    assert abs(cosine[:, 2].mean() - 2 / 3) < 0.006
    for b in range(4):
        lo, hi = b / 4, (b + 1) / 4
        check_frequency(int(np.sum(np.minimum((r2 * 4).astype(int), 3) == b)), 0.25, count)
        check_frequency(int(np.sum(np.minimum((cosine[:, 2] * 4).astype(int), 3) == b)),
                        hi * hi - lo * lo, count)
    tri = oracle.warp("triangle", u)
    assert np.allclose(tri.sum(1), 1, atol=1e-12)
    assert np.all(np.abs(tri.mean(0) - 1 / 3) < 0.006)
    assert abs((tri[:, 0] * tri[:, 1]).mean() - 1 / 12) < 0.002
    assert np.array_equal(oracle.warp("disk", [0.5, 0.5])[0, :2], [0, 0])
    with pytest.raises(oracle.OracleError):
        oracle.warp("sphere", [1.0, 0.0])
    with pytest.raises(oracle.OracleError):
        oracle.warp("disk", [0.0, -0.1])


def test_discrete_distribution_known_answers(oracle):
    # tests/sampling_tests.cpp:140-173
    prob, idx, mass, remap = oracle.distribution([0, 1, 3, 0],
                                                 [0, 0.25, np.nextafter(1.0, 0.0)])
    assert prob[0] == 0 and prob[3] == 0
    assert prob[1] == pytest.approx(0.25) and prob[2] == pytest.approx(0.75)
    assert idx.tolist() == [1, 2, 2]
    us = oracle.stream_1d(41, 0, 0, 20000)
    prob, idx, mass, remap = oracle.distribution([0, 1, 3, 0], us)
    assert np.all((remap >= 0) & (remap < 1))
    check_frequency(int(np.sum(idx == 1)), 0.25, len(us))
    assert oracle.distribution([0, 0, 0], [0.5])[0][1] == pytest.approx(1 / 3)
    assert oracle.distribution([1e308, 1e308], [0.5])[0][0] == pytest.approx(0.5)
    with pytest.raises(oracle.OracleError):
        oracle.distribution([-1.0], [0.5])
    with pytest.raises(oracle.OracleError):
        oracle.distribution([0, 1, 3, 0], [1.0])


# ---- BSDF (tests/sampling_tests.cpp:187-407) ----

def test_lambert_weight_equals_albedo(oracle):
    # tests/sampling_tests.cpp:187-215 (texture colour folded into the base colour)
    wo = np.array([0.5, 0.1, 1.0]) / np.linalg.norm([0.5, 0.1, 1.0])
    color = (0.4, 0.4, 0.0)
    us = oracle.stream_1d(4, 0, 0, 3 * 500).reshape(-1, 3)
    for c, u0, u1 in us:
        s = oracle.bsdf_sample("diffuse", wo, c, [u0, u1], base_color=color)
        assert s is not None and not s["discrete"]
        assert np.linalg.norm(s["weight"] - np.array(color, np.float32)) < 1e-7
        value, pdf, _ = oracle.bsdf_eval("diffuse", wo, s["direction"], base_color=color)
        assert s["probability"] == pytest.approx(pdf, rel=1e-12)
        assert np.linalg.norm(value * s["direction"][2] / s["probability"] - s["weight"]) < 1e-12
    assert oracle.bsdf_sample("diffuse", [0, 0, -1], 0.5, [0.5, 0.5]) is None


def test_ggx_null_event_probability_and_albedo(oracle):
    # tests/sampling_tests.cpp:217-255
    count = 20000
    wo = [0.0, 0.0, 1.0]
    for roughness in (0.4, 0.7, 1.0):
        us = oracle.stream_1d(87, 0, 0, 3 * count).reshape(-1, 3)
        nulls = 0
        albedo = 0.0
        for c, u0, u1 in us:
            s = oracle.bsdf_sample("conductor", wo, c, [u0, u1], roughness=roughness)
            if s is None:
                nulls += 1
                continue
            albedo += s["weight"][0]
        alpha = np.float32(roughness) ** 2
        a2 = float(alpha) ** 2
        u = lambda z: (1 - z) / (1 + a2 + (a2 - 1) * z)  # noqa: E731
        check_frequency(nulls, 1 - u(0), count)
        if roughness == 1.0:
            assert albedo / count == pytest.approx(1 - math.log(2.0), abs=0.01)
            quadrature = 0.0
            for row in range(512):
                z = (row + 0.5) / 512
                v, _, _ = oracle.bsdf_eval("conductor", wo, [math.sqrt(1 - z * z), 0, z],
                                           roughness=1.0)
                quadrature += v[0] * z * 2 * PI / 512
            assert quadrature == pytest.approx(1 - math.log(2.0), abs=1e-6)


def test_mirror_and_smooth_conductor_are_discrete(oracle):
    # tests/sampling_tests.cpp:320-340
    wo = np.array([0.6, 0.0, 0.8])
    for kind in ("mirror", "conductor"):
        s = oracle.bsdf_sample(kind, wo, 0.2, [0.3, 0.4], base_color=(0.9, 0.7, 0.3),
                               roughness=0.0)
        assert s["discrete"] and s["probability"] == 1
        assert np.linalg.norm(s["direction"] - [-wo[0], -wo[1], wo[2]]) < 1e-12
        v, pdf, delta = oracle.bsdf_eval(kind, wo, s["direction"], roughness=0.0)
        assert delta and pdf == 0 and np.all(v == 0)


def test_dielectric_fresnel_snell_and_tir(oracle):
    # tests/sampling_tests.cpp:342-407
    assert oracle.fresnel_dielectric(1, 1, 1.5) == pytest.approx(0.04)
    assert oracle.fresnel_dielectric(0, 1, 1.5) == 1
    assert oracle.fresnel_dielectric(0, 1, 1) == 0
    assert oracle.fresnel_dielectric(0.5, 1.5, 1) == 1
    wo = np.array([0.6, 0.0, 0.8])
    reflected = oracle.bsdf_sample("dielectric", wo, 0.0, [0.5, 0.5])
    transmitted = oracle.bsdf_sample("dielectric", wo, 0.99, [0.5, 0.5])
    importance = oracle.bsdf_sample("dielectric", wo, 0.99, [0.5, 0.5], importance=True)
    assert reflected["event"] == 2 and transmitted["event"] == 3
    assert transmitted["discrete"]
    assert transmitted["direction"][0] == pytest.approx(-wo[0] / 1.5)
    assert transmitted["direction"][2] < 0
    assert transmitted["eta"] == pytest.approx(1.5)
    assert transmitted["weight"][0] == pytest.approx(1 / 2.25)
    assert importance["weight"][0] == 1
    assert reflected["probability"] + transmitted["probability"] == pytest.approx(1)
    exit_ = oracle.bsdf_sample("dielectric", -transmitted["direction"], 0.99, [0.5, 0.5],
                               front_face=False)
    assert transmitted["weight"][0] * exit_["weight"][0] == pytest.approx(1)
    tir = oracle.bsdf_sample("dielectric", np.array([0.9, 0, 0.3]) / np.linalg.norm([0.9, 0, 0.3]),
                             0.999, [0.2, 0.5], front_face=False)
    assert tir["event"] == 2 and tir["probability"] == 1 and np.all(tir["weight"] == 1)
    matched = oracle.bsdf_sample("dielectric", wo, 0.0, [0.0, 0.0], ior=1.0)
    assert matched["probability"] == 1
    assert np.linalg.norm(matched["direction"] + wo) < 1e-12
    with pytest.raises(oracle.OracleError):
        oracle.fresnel_dielectric(0.5, -1, 1)


def test_power_heuristic_limits(oracle):
    # tests/path_tests.cpp:122-132
    assert oracle.power_heuristic(1, 1) == 0.5
    assert oracle.power_heuristic(1e300, 1e300) == 0.5
    assert oracle.power_heuristic(3, 4) == pytest.approx(9 / 25)
    assert oracle.power_heuristic(0, 1) == 0
    assert oracle.power_heuristic(1, 0) == 1
    assert oracle.power_heuristic(0, 0) == 0
    with pytest.raises(oracle.OracleError):
        oracle.power_heuristic(-1, 1)


# ---- lights (tests/light_tests.cpp) ----

def area_scene():
    """One emissive triangle (-1,-1,0),(1,-1,0),(-1,1,0) with radiance (4,2,1)
    (tests/light_tests.cpp:40-51)."""
    doc = SceneDocument(environment=(0.0, 0.0, 0.0))
    doc.meshes.append(MeshData(np.array([[-1, -1, 0], [1, -1, 0], [-1, 1, 0]], np.float32),
                               np.array([[0, 1, 2]], np.uint32),
                               np.tile(np.array([0, 0, 1], np.float32), (1, 3, 1))))
    doc.materials.append(Material(emission=(4.0, 2.0, 1.0)))
    doc.objects.append(SceneObject(0, 0))
    return doc


def test_area_light_pdf_known_answer(oracle):
    # tests/light_tests.cpp:165-191
    o = oracle.OracleScene(area_scene().snapshot())
    s = o.light_sample([0, 0, 2], 0.5, [0.25, 0.5])
    assert s["kind"] == 0 and not s["discrete"]
    assert s["distance"] == pytest.approx(math.sqrt(4.5))
    assert s["probability"] == pytest.approx(4.5 ** 1.5 / 4)
    assert np.array_equal(s["radiance"], [4, 2, 1])
    below = o.light_sample([0, 0, -2], 0.5, [0.25, 0.5])
    assert below["probability"] == pytest.approx(s["probability"])


def test_light_selection_pmfs(oracle):
    # tests/light_tests.cpp:193-235
    doc = area_scene()
    doc.objects.append(SceneObject(0, 0, Transform((3.0, 0.0, 0.0), (0, 0, 0), (2.0, 2.0, 1.0))))
    doc.directional_lights.append(DirectionalLight((0, -2, 0), (1, 1, 1), 2.0))
    doc.environment = (0.25, 0.25, 0.25)
    o = oracle.OracleScene(doc.snapshot())
    le = 4 * 0.2126 + 2 * 0.7152 + 1 * 0.0722
    powers = np.array([4 * PI * le, 16 * PI * le, 26 * PI, 13 * PI * PI])
    masses = powers / powers.sum()
    assert np.allclose(o.light_probabilities(), masses, rtol=1e-12)
    cdf = 0.0
    for i, m in enumerate(masses):
        s = o.light_sample([0, 0, 2], cdf + m * 0.5, [0.3, 0.4])
        assert s["emitter"] == i
        if i == 2:
            assert s["discrete"] and np.array_equal(s["direction"], [0, 1, 0])
            assert np.array_equal(s["radiance"], [2, 2, 2])
            assert s["probability"] == pytest.approx(m)
        if i == 3:
            assert s["kind"] == 2 and s["probability"] == pytest.approx(m / (4 * PI))
        cdf += m
    empty = oracle.OracleScene(SceneDocument(environment=(0.0, 0.0, 0.0)).snapshot())
    assert len(empty.light_probabilities()) == 0
    assert empty.light_sample([0, 0, 0], 0.4, [0.5, 0.5]) is None


# ---- intersection + BVH (tests/intersection_tests.cpp) ----

def triangle_doc(vertices=((0, 0, 0), (1, 0, 0), (0, 1, 0)), double_sided=True):
    doc = SceneDocument()
    doc.meshes.append(MeshData(np.array(vertices, np.float32), np.array([[0, 1, 2]], np.uint32),
                               np.tile(np.array([0, 0, 1], np.float32), (1, 3, 1))))
    doc.materials.append(Material(double_sided=double_sided))
    doc.objects.append(SceneObject(0, 0))
    return doc


def test_shear_test_barycentrics_and_closed_interval(oracle):
    # tests/intersection_tests.cpp:143-159
    o = oracle.OracleScene(triangle_doc(((0, 0, 0), (2, 0, 0), (0, 2, 0))).snapshot())
    hit, _ = o.intersect([[0.5, 0.5, 2]], [[0, 0, -1]], 0, 10)
    assert hit[0, 0] == 1 and hit[0, 1] == pytest.approx(2)
    assert hit[0, 5:8] == pytest.approx([0.5, 0.25, 0.25])
    assert o.intersect([[0.5, 0.5, 2]], [[0, 0, -1]], 2, 2)[0][0, 0] == 1
    assert o.intersect([[0.5, 0.5, 2]], [[0, 0, -1]], 0, 1.99)[0][0, 0] == 0
    assert o.intersect([[0.5, 0.5, 2]], [[0, 0, -1]], 2.01, 10)[0][0, 0] == 0
    assert o.intersect([[0.5, 0.5, -2]], [[0, 0, 1]], 0, 10)[0][0, 0] == 1
    assert o.intersect([[3, 3, 2]], [[0, 0, -1]], 0, 10)[0][0, 0] == 0


def studio_cubes():
    """30 transformed single-sided cubes (tests/intersection_tests.cpp:264-281)."""
    doc = SceneDocument()
    doc.materials.append(Material("diffuse", (0.05, 0.3, 0.65), double_sided=False))
    doc.meshes.append(box_mesh((1, 1, 1)))
    for z in range(5):
        for x in range(6):
            t = Transform((float(x * 2 - 5), 0.0, float(z * 2 - 4)),
                          (float(x * 7), float(z * 11), 0.0),
                          (-0.7 if x % 2 else 0.7, 0.6 + z * 0.1, 1.0))
            doc.objects.append(SceneObject(0, 0, t))
    return doc


def lcg_rays(count=4000):
    """The fixed LCG ray set of tests/intersection_tests.cpp:105-108,286-293."""
    state = 0x12345678

    def rnd():
        nonlocal state
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        return np.float32(state >> 8) / np.float32(8388608.0) - np.float32(1)

    origins, targets = [], []
    for _ in range(count):
        o = [rnd() * np.float32(8), np.float32(3) + rnd(), rnd() * np.float32(8)]
        t = [rnd() * np.float32(7), rnd(), rnd() * np.float32(7)]
        origins.append(o)
        targets.append(t)
    origins = np.array(origins, np.float32)
    targets = np.array(targets, np.float32)
    d = (targets - origins).astype(np.float32)
    d = d * (np.float32(1) / np.sqrt((d * d).sum(1, dtype=np.float32)))[:, None]
    return origins.astype(np.float32), d.astype(np.float32)


def brute_force(tris, single_sided_mirror, o, d, tmin, tmax):
    """Independent double Moller-Trumbore (tests/intersection_tests.cpp:72-102)."""
    v0, v1, v2 = (tris[:, k].astype(np.float64) for k in range(3))
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(d, e2)
    det = (e1 * p).sum(1)
    ok = np.abs(det) >= 1e-14
    ss, mir = single_sided_mirror
    ok &= ~(ss & (det * np.where(mir, -1, 1) <= 0))
    with np.errstate(divide="ignore", invalid="ignore"):
        off = o - v0
        u = (off * p).sum(1) / det
        q = np.cross(off, e1)
        v = (d * q).sum(1) / det
        t = (e2 * q).sum(1) / det
    ok &= (u >= 0) & (v >= 0) & (u + v <= 1) & (t >= tmin) & (t <= tmax)
    if not ok.any():
        return None
    i = int(np.argmin(np.where(ok, t, np.inf)))
    return i, t[i]


def test_bvh_matches_brute_force_on_lcg_rays(oracle):
    # tests/intersection_tests.cpp:264-311
    snap = studio_cubes().snapshot()
    o = oracle.OracleScene(snap)
    tris = o.primitives()
    n = len(tris)
    mirrored = np.repeat([np.linalg.det(m[:3, :3].astype(np.float64)) < 0
                          for m, _ in snap.matrices], 12)
    single = np.ones(n, bool)
    origins, dirs = lcg_rays()
    tmax = np.where(np.arange(4000) % 2 == 1, 100.0, 3.0)
    hits, counters = o.intersect(origins, dirs, 1e-5, tmax)
    occ, _ = o.occluded(origins, dirs, 1e-5, tmax)
    found = 0
    for i in range(4000):
        ref = brute_force(tris, (single, mirrored), origins[i].astype(np.float64),
                          dirs[i].astype(np.float64), 1e-5, tmax[i])
        assert (hits[i, 0] == 1) == (ref is not None)
        assert occ[i] == (ref is not None)
        if ref is not None:
            found += 1
            assert hits[i, 1] == pytest.approx(ref[1], abs=1e-7)
            assert int(hits[i, 4]) == ref[0]
    assert found > 300
    assert counters[1] < n * 4000


def test_coincident_centroids_and_any_hit_early_exit(oracle):
    # tests/intersection_tests.cpp:313-336
    doc = triangle_doc()
    for _ in range(255):
        doc.objects.append(SceneObject(0, 0))
    o = oracle.OracleScene(doc.snapshot())
    assert o.bvh_counts()["nodes"] == 1
    hit, nearest = o.intersect([[0.25, 0.25, 2]], [[0, 0, -1]])
    assert hit[0, 2] == 0
    occ, shadow = o.occluded([[0.25, 0.25, 2]], [[0, 0, -1]])
    assert occ[0] and nearest[1] == 256 and shadow[1] == 1
    assert not o.occluded([[0.25, 0.25, 2]], [[0, 0, -1]], 0, 1.9)[0][0]
    with pytest.raises(oracle.OracleError):
        o.intersect([[0.25, 0.25, 2]], [[0, 0, -1]], 3, 2)


def test_bvh_prunes_separated_triangles(oracle):
    # tests/intersection_tests.cpp:350-379
    doc = triangle_doc()
    doc.objects = [SceneObject(0, 0, Transform((x * 2.0, 0.0, 0.0))) for x in range(64)]
    o = oracle.OracleScene(doc.snapshot())
    origins = [[x * 2 + 0.25, 0.25, 2] for x in range(64)]
    hits, counters = o.intersect(origins, [[0, 0, -1]] * 64)
    assert np.array_equal(hits[:, 2], np.arange(64))
    assert counters[1] <= 64 * 4


def test_single_sided_culling(oracle):
    # tests/sided_tests.cpp:54-90
    for double_sided in (False, True):
        o = oracle.OracleScene(triangle_doc(double_sided=double_sided).snapshot())
        front, _ = o.intersect([[0.2, 0.2, 2]], [[0, 0, -1]])
        back, _ = o.intersect([[0.2, 0.2, -2]], [[0, 0, 1]])
        assert front[0, 0] == 1 and front[0, 8] == 1
        assert back[0, 0] == (1 if double_sided else 0)


# ---- integrator (tests/path_tests.cpp) ----

def emitter_doc():
    """tests/path_tests.cpp:23-34"""
    doc = SceneDocument(environment=(0.0, 0.0, 0.0))
    doc.meshes.append(MeshData(np.array([[-1, -1, 0], [1, -1, 0], [-1, 1, 0]], np.float32),
                               np.array([[0, 1, 2]], np.uint32),
                               np.tile(np.array([0, 0, 1], np.float32), (1, 3, 1))))
    doc.materials.append(Material(emission=(1.0, 1.0, 1.0)))
    doc.objects.append(SceneObject(0, 0))
    return doc


def floor_doc(kind="diffuse", color=0.6):
    """tests/path_tests.cpp:36-52"""
    doc = SceneDocument(environment=(1.0, 1.0, 1.0))
    doc.camera = Camera(position=(0.0, 1.0, 0.0), target=(0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0))
    doc.meshes.append(quad_mesh([(-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)], (0, 1, 0)))
    doc.materials.append(Material(kind, (color, color, color)))
    doc.objects.append(SceneObject(0, 0, Transform(scale=(4.0, 1.0, 4.0))))
    return doc


def direct_doc(glossy):
    """tests/path_tests.cpp:56-67"""
    doc = floor_doc("conductor" if glossy else "diffuse", 0.8 if glossy else 0.7)
    doc.environment = (0.0, 0.0, 0.0)
    doc.materials[0].roughness = 0.15
    e = 1.0 if glossy else 16.0
    doc.materials.append(Material(emission=(e, e, e)))
    doc.objects.append(SceneObject(0, 1, Transform((0.0 if glossy else 0.75, 2.0, 0.0), (0, 0, 0),
                                                   (2.5 if glossy else 0.125, 1.0,
                                                    2.5 if glossy else 0.125))))
    return doc


def estimate(o, count, seed, origin=(0, 1, 0), direction=(0, -1, 0), interval=(0, 10000)):
    keys = np.zeros((count, 3), np.uint64)
    keys[:, 0] = seed
    keys[:, 2] = np.arange(count)
    rad, stats = o.trace_paths([origin] * count, [direction] * count, interval[0], interval[1],
                               keys)
    x = rad[:, 0]
    return x.mean(), x.std(ddof=1) / math.sqrt(count), stats


def sampler_doubles(oracle, seed, count, sequence=1):
    """Sampler(seed, sequence).next_1d() values (src/core/sampling.cpp:56-60)."""
    raw = oracle.pcg_sequence(seed, sequence, 2 * count).astype(np.uint64)
    hi = raw[0::2] >> np.uint64(5)
    lo = raw[1::2] >> np.uint64(6)
    return (hi.astype(np.float64) * 67108864.0 + lo.astype(np.float64)) / 9007199254740992.0


def test_false_endpoint_occlusions(oracle):
    # tests/path_tests.cpp:103-120
    o = oracle.OracleScene(emitter_doc().snapshot())
    seq = sampler_doubles(oracle, 171, 2000).reshape(-1, 2)
    origin = np.array([0.5, 0.25, 4.0])
    false = 0
    for i in range(1000):
        s = o.light_sample(origin, 0.5, seq[i])
        occ, _ = o.occluded([origin], [s["direction"]], 0, s["distance"] * (1 - 1e-9))
        false += int(occ[0])
    assert false == 0


@pytest.mark.parametrize("mode", ["bsdf", "light", "mis"])
def test_diffuse_constant_environment(oracle, mode):
    # tests/path_tests.cpp:134-158
    o = oracle.OracleScene(floor_doc().snapshot(), oracle.integrator(mode, 1, False, 3))
    mean, se, _ = estimate(o, 8192, 81)
    assert abs(mean - np.float32(0.6)) < 5 * se + 1e-8


def test_diffuse_albedo_exact_across_scales(oracle):
    # tests/path_tests.cpp:150-157
    for scale in (0.001, 1.0, 1000.0):
        doc = floor_doc()
        s = np.float32(scale)
        doc.objects[0].transform = Transform((s * 7, s * 7, s * 7), (0, 0, 0), (4 * s, s, 4 * s))
        o = oracle.OracleScene(doc.snapshot(), oracle.integrator("bsdf", 1, False, 3))
        keys = np.array([[31, 0, 0]], np.uint64)
        rad, _ = o.trace_paths([[s * 7, s * 8, s * 7]], [[0, -1, 0]], 0, 10000, keys)
        assert rad[0, 0] == pytest.approx(float(np.float32(0.6)), abs=1e-8)


@pytest.mark.parametrize("mode", ["bsdf", "light", "mis"])
def test_directional_light_exact(oracle, mode):
    # tests/path_tests.cpp:160-172
    doc = floor_doc()
    doc.environment = (0.0, 0.0, 0.0)
    irradiance = float(np.float32(PI))
    doc.directional_lights.append(DirectionalLight((0, -1, 0), (1, 1, 1), irradiance))
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator(mode, 1, False, 3))
    mean, _, _ = estimate(o, 32, 3)
    assert mean == pytest.approx(float(np.float32(0.6)) * irradiance / PI, abs=1e-10)


@pytest.mark.parametrize("mode", ["bsdf", "light", "mis"])
def test_mirror_and_glass_exact(oracle, mode):
    # tests/path_tests.cpp:174-190
    o = oracle.OracleScene(floor_doc("mirror", 0.7).snapshot(), oracle.integrator(mode, 2, False, 3))
    assert estimate(o, 128, 9)[0] == pytest.approx(float(np.float32(0.7)), abs=1e-10)
    glass = floor_doc("dielectric", 1.0)
    glass.objects.append(SceneObject(0, 0, Transform((0.0, -1.0, 0.0), (180.0, 0.0, 0.0),
                                                     (4.0, 1.0, 4.0))))
    o = oracle.OracleScene(glass.snapshot(), oracle.integrator(mode, 12, False, 3))
    assert estimate(o, 1024, 125)[0] == pytest.approx(1.0, abs=1e-8)


def test_depth_zero_returns_emission(oracle):
    # tests/path_tests.cpp:192-205
    doc = floor_doc()
    doc.environment = (0.0, 0.0, 0.0)
    doc.materials[0].emission = (8.0, 2.0, 0.5)
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator("mis", 0, False, 3))
    rad, stats = o.trace_paths([[0, 1, 0]], [[0, -1, 0]], 0, 100, np.array([[9, 0, 0]], np.uint64))
    assert rad[0].tolist() == [8, 2, 0.5]
    assert stats["scattering_events"] == 0 and stats["shadow_rays"] == 0


def test_russian_roulette_mean(oracle):
    # tests/path_tests.cpp:207-228
    doc = floor_doc("diffuse", 0.5)
    doc.environment = (0.0, 0.0, 0.0)
    doc.materials[0].emission = (1.0, 1.0, 1.0)
    doc.objects[0].transform = Transform(scale=(1000.0, 1.0, 1000.0))
    doc.objects.append(SceneObject(0, 0, Transform((0.0, 2.0, 0.0), (0, 0, 0),
                                                   (1000.0, 1.0, 1000.0))))
    snap = doc.snapshot()
    no_rr = oracle.OracleScene(snap, oracle.integrator("bsdf", 8, False, 1))
    rr = oracle.OracleScene(snap, oracle.integrator("bsdf", 8, True, 1))
    m0, e0, s0 = estimate(no_rr, 4096, 13)
    m1, e1, s1 = estimate(rr, 16384, 14)
    assert abs(m1 - m0) < 5 * math.hypot(e0, e1) + 0.002
    assert m0 == pytest.approx(2 - 1 / 256, abs=0.003)
    assert s1["roulette_terminations"] > 0
    assert s1["scattering_events"] / s1["paths"] < s0["scattering_events"] / s0["paths"]


def test_blocker_in_front_and_behind_light(oracle):
    # tests/path_tests.cpp:267-289
    doc = direct_doc(False)
    clear = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    doc.materials.append(Material(base_color=(0.0, 0.0, 0.0)))
    blocker = SceneObject(0, 2, Transform((0.0, 1.0, 0.0), (0, 0, 0), (4.0, 1.0, 4.0)))
    doc.objects.append(blocker)
    blocked = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    blocker.transform = Transform((0.0, 3.0, 0.0), (0, 0, 0), (4.0, 1.0, 4.0))
    behind = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    keys = np.zeros((256, 3), np.uint64)
    keys[:, 0] = 79
    keys[:, 2] = np.arange(256)
    args = ([[0, 0.5, 0]] * 256, [[0, -1, 0]] * 256, 0, np.inf, keys)
    a, _ = clear.trace_paths(*args)
    b, _ = blocked.trace_paths(*args)
    c, _ = behind.trace_paths(*args)
    assert np.all(a[:, 0] > 0) and np.all(b == 0)
    assert np.max(np.linalg.norm(c - a, axis=1)) < 1e-12


def test_translation_invariance(oracle):
    # tests/path_tests.cpp:251-265
    doc = direct_doc(False)
    original = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    for obj in doc.objects:
        t = obj.transform
        obj.transform = Transform(tuple(np.float32(v) * np.float32(128) + np.float32(1e8)
                                        for v in t.translation), t.rotation_degrees,
                                  tuple(np.float32(v) * np.float32(128) for v in t.scale))
    moved = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    keys = np.zeros((512, 3), np.uint64)
    keys[:, 0] = 5
    keys[:, 2] = np.arange(512)
    a, _ = original.trace_paths([[0, 1, 0]] * 512, [[0, -1, 0]] * 512, 0, np.inf, keys)
    b, _ = moved.trace_paths([[1e8, 1e8 + 128, 1e8]] * 512, [[0, -1, 0]] * 512, 0, np.inf, keys)
    assert np.max(np.linalg.norm(a - b, axis=1)) < 1e-7


def test_thin_lens_focus_plane(oracle):
    # tests/path_tests.cpp:230-249, through sample_pixel's camera ray: every lens ray passes
    # through the focus point of the pinhole ray with the same film position.
    doc = SceneDocument(environment=(0.0, 0.0, 0.0))
    doc.camera = Camera(position=(0.0, 0.0, 5.0), target=(0.0, 0.0, 0.0), aperture_radius=0.2,
                        focus_distance=3.0)
    o = oracle.OracleScene(doc.snapshot())
    w, h = 8, 6
    render = _abi.RenderSettings(w, h, 16, 3)
    _, _, rays = o.sample_pixels(render, [[5, 2]] * 16, np.arange(16), want_rays=True)
    half = math.tan(math.radians(45.0) * 0.5)
    for s in range(16):
        film = oracle.stream_1d(3, 2 * w + 5, s, 2)
        u, v = (5 + film[0]) / w, (2 + film[1]) / h
        d = np.array([0, 0, -1.0]) + (2 * u - 1) * (w / h) * half * np.array([1.0, 0, 0]) \
            + (1 - 2 * v) * half * np.array([0, 1.0, 0])
        d /= np.linalg.norm(d)
        focus = np.array([0, 0, 5.0]) + d * (3 / -d[2])
        t = (focus[2] - rays[s, 2]) / rays[s, 5]
        point = rays[s, 0:3] + rays[s, 3:6] * t
        assert np.linalg.norm(point - focus) < 1e-12
        assert np.linalg.norm(rays[s, 0:3] - [0, 0, 5]) <= 0.2 + 1e-7
        assert abs(np.linalg.norm(rays[s, 3:6]) - 1) < 1e-12


def test_render_threads_bitwise_equal_and_sample_pixel_mean(oracle):
    # tests/session_tests.cpp:87-123 and tests/path_tests.cpp:360-378
    from minirender_b200.scene import cornell_box
    o = oracle.OracleScene(cornell_box().snapshot(), oracle.integrator("mis", 4, False, 3))
    render = _abi.RenderSettings(17, 13, 9, 413)
    serial, _ = o.render(render, threads=1)
    for threads in (3, 4):
        parallel, _ = o.render(render, threads=threads)
        assert np.array_equal(serial, parallel)
    rad, _ = o.sample_pixels(render, [[1, 1]] * 9, np.arange(9))
    assert np.array_equal(serial[1, 1], (rad.sum(0) / 9).astype(np.float32))


def test_display_image_reinhard(oracle):
    # tests/path_tests.cpp:374-377
    d = oracle.display_image(np.array([[[8, 2, 0.5]]], np.float32))
    assert d[0, 0, 0] == pytest.approx(8 / 9, abs=1e-7)
    assert oracle.display_image(np.array([[[8, 2, 0.5]]], np.float32), 2)[0, 0, 1] > d[0, 0, 1]


# ---- media (tests/medium_tests.cpp, tests/volume_path_tests.cpp) ----

def test_hg_normalisation_and_symmetry(oracle):
    # tests/medium_tests.cpp:64-80
    wo = [0, 0, 1]
    for g in (-0.9, -0.4, 0.0, 0.4, 0.9):
        c, weights = np.polynomial.legendre.leggauss(256)
        vals = np.array([2 * PI * oracle.phase(wo, [math.sqrt(max(0, 1 - x * x)), 0, -x], g)
                         for x in c])
        assert np.dot(weights, vals) == pytest.approx(1, abs=2e-9)
        assert np.dot(weights, c * vals) == pytest.approx(g, abs=2e-9)
    wi = np.array([0.3, -0.4, 0.7]) / np.linalg.norm([0.3, -0.4, 0.7])
    assert oracle.phase(wo, wi, 0.3) == oracle.phase(wi, wo, 0.3)
    assert oracle.phase(wo, wi, 0.0) == pytest.approx(1 / (4 * PI), rel=1e-14)


def test_free_flight_zero_channel_and_vacuum(oracle):
    # tests/medium_tests.cpp:160-178
    scattered, _, w = oracle.medium_distance([0, 0.2, 0.3], [0, 0.5, 0.9], 4, 0.1, 0.5)
    assert not scattered
    tr = np.exp(-np.array([0, 0.7, 1.2]) * 4)
    assert np.allclose(w, tr * (3 / tr.sum()), rtol=1e-12)
    scattered, _, w = oracle.medium_distance([0, 0, 0], [0, 0, 0], 4, 0.5, 0.9)
    assert not scattered and np.allclose(w, 1)


def test_volume_absorption_within_clip_interval(oracle):
    # tests/volume_path_tests.cpp:93-105
    from minirender_b200.scene import MediumRegion
    doc = SceneDocument(environment=(1.0, 1.0, 1.0))
    doc.camera = Camera(position=(-2.0, 0.0, 0.0), target=(0.0, 0.0, 0.0), near_plane=0.01)
    doc.media = [MediumRegion((-1, -1, -1), (1, 1, 1), (0.1, 0.4, 0.8), (0, 0, 0), 0.0)]
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator("mis", 0, True, 3))
    rad, _ = o.trace_paths([[-2, 0, 0]], [[1, 0, 0]], 1.25, 2.75, np.array([[77, 0, 0]], np.uint64))
    expected = np.exp(-np.array([0.1, 0.4, 0.8]) * 1.5)
    assert np.linalg.norm(rad[0] - expected) < 1e-12
