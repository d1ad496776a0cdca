"""Two-level scenes (an instance tree over one object-space tree per mesh) against the flattened
world-space tree the reference builds (src/render/bvh.cpp:31-99).

The two-level traversal tests every candidate triangle in world space with the flattening's own
vertex arithmetic, so the bar is exact: nearest hits (primitive, distance, barycentrics, instance,
triangle, facing) and occlusion equal the flattened scene's bit for bit, images and the path
counters other than the traversal counters are bitwise equal, in the plain path and in batched
waves that mix both kinds of scene. A refit (new instance transforms, new mesh positions) renders
exactly like a scene built from the updated description. A mesh instanced many times is stored
once: the job scenes of the batching workload (8 meshes instanced tens of times) take a fraction
of the flattened scene's device memory.
"""

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


def mirrored_and_scaled():
    """Instances with mirrored, non-uniformly scaled and rotated transforms, one far from the
    origin, over a ground quad, lit by the environment and a directional light."""
    doc = sc.sphere_field(12, 6.0, 4, subdivisions=2, variants=3)
    doc.objects[1].transform = sc.Transform((1.0, 2.0, -1.0), (10.0, 20.0, 30.0), (-1.0, 0.5, 2.0))
    doc.objects[2].transform = sc.Transform((-2.0, 1.5, 0.5), (0.0, 45.0, 0.0), (3.0, 0.25, 1.0))
    doc.objects[3].transform = sc.Transform((5000.0, 3000.0, -7000.0), (0, 0, 0), (1.0, 1.0, 1.0))
    return doc


SCENES = {
    "cornell": sc.cornell_box,
    "room": lambda: sc.job_scene(60_000, 12),
    "spheres": lambda: sc.sphere_field(40, 10.0, 9, 3, variants=5),
    "transforms": mirrored_and_scaled,
    # more instances than one 128-thread block of the per-instance kernels
    "many": lambda: sc.sphere_field(700, 40.0, 13, 1, variants=6),
}


def rays(doc, n, seed):
    """Rays from points around the scene's middle towards random points, and camera-like rays."""
    rng = np.random.default_rng(seed)
    snap = doc.snapshot()
    tris = snap.world_triangles().reshape(-1, 3)
    lo, hi = np.percentile(tris, 2, axis=0), np.percentile(tris, 98, axis=0)
    origins = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    targets = tris[rng.integers(0, len(tris), n)] + rng.normal(0, 0.05, (n, 3))
    d = targets - origins
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return origins, d


def assert_same_hits(a, b):
    for key in a.dtype.names:
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


@pytest.mark.parametrize("name", list(SCENES))
def test_two_level_hits_equal_flattened(api, name):
    doc = SCENES[name]()
    snap = doc.snapshot()
    flat = api.Scene(snap)
    two = api.Scene(snap, two_level=True)
    o, d = rays(doc, 200_000, 3)
    ha, _ = flat.intersect(o, d, 0.0, np.inf)
    hb, sb = two.intersect(o, d, 0.0, np.inf)
    assert (ha["primitive"] != 0xFFFFFFFF).mean() > 0.3
    assert_same_hits(ha, hb)
    for tmax in (0.5, 3.0):
        oa, _ = flat.occluded(o, d, 1e-4, tmax)
        ob, _ = two.occluded(o, d, 1e-4, tmax)
        np.testing.assert_array_equal(oa, ob)
    assert sb["triangle_tests"] > 0


@pytest.mark.parametrize("name", ["cornell", "room", "spheres", "transforms"])
def test_two_level_images_equal_flattened(api, name):
    doc = SCENES[name]()
    snap = doc.snapshot()
    settings = api.IntegratorSettings("mis", 8, True, 3)
    render = api.RenderSettings(96, 72, 8, 5)
    img_a, st_a = api.PathTracer(api.Scene(snap), settings).render(render)
    img_b, st_b = api.PathTracer(api.Scene(snap, two_level=True), settings).render(render)
    np.testing.assert_array_equal(img_a, img_b)
    for key in ("paths", "shadow_rays", "scattering_events", "roulette_terminations"):
        assert st_a[key] == st_b[key], key
    assert img_a.mean() > 0


def test_two_level_scene_in_a_mixed_batch(api):
    a_doc, b_doc = sc.job_scene(30_000, 7), sc.sphere_field(20, 6.0, 2, 2, variants=3)
    settings = api.IntegratorSettings("mis", 6, True, 3)
    jobs, alone = [], []
    for doc, two_level, render in ((a_doc, True, api.RenderSettings(64, 64, 6, 1)),
                                   (b_doc, False, api.RenderSettings(48, 40, 5, 2)),
                                   (b_doc, True, api.RenderSettings(40, 48, 7, 3))):
        scene = api.Scene(doc.snapshot(), two_level=two_level)
        jobs.append(api.BatchJob(scene, render, settings))
        alone.append(api.PathTracer(api.Scene(doc.snapshot()), settings).render(render)[0])
    images, codes, _ = api.render_batch(jobs, api.BatchSettings(wave_paths=8192))
    assert codes == [0, 0, 0]
    for got, want in zip(images, alone):
        np.testing.assert_array_equal(got, want)


def test_instanced_mesh_is_stored_once(api):
    doc = sc.job_scene(300_000, 11)  # 8 displaced meshes instanced into ~300k triangles
    snap = doc.snapshot()
    flat = api.Scene(snap)
    two = api.Scene(snap, two_level=True)
    print(f"device bytes: flattened {flat.device_bytes()}, two-level {two.device_bytes()}")
    assert two.device_bytes() * 5 < flat.device_bytes()
    st = two.statistics()
    assert st["triangles"] == snap.triangle_count


def moved(doc, k):
    out = sc.SceneDocument(**{f: getattr(doc, f) for f in doc.__dataclass_fields__})
    out.objects = list(doc.objects)
    for i in range(k, len(out.objects)):
        t = out.objects[i].transform
        out.objects[i] = sc.SceneObject(out.objects[i].mesh, out.objects[i].material,
                                        sc.Transform(tuple(v + 0.03 * (i % 3) for v in t.translation),
                                                     tuple(r + 7.0 for r in t.rotation_degrees),
                                                     t.scale), out.objects[i].visible)
    return out


def test_update_instances_renders_like_a_fresh_build(api):
    doc = sc.job_scene(40_000, 21)  # the Cornell shell (walls, boxes, light) first, then spheres
    first = 8                       # the spheres: none of them emits
    two = api.Scene(doc.snapshot(), two_level=True)
    after = moved(doc, first)
    two.update_instances(first, after)
    fresh = api.Scene(after.snapshot())
    o, d = rays(after, 100_000, 9)
    assert_same_hits(fresh.intersect(o, d, 0.0, np.inf)[0], two.intersect(o, d, 0.0, np.inf)[0])
    settings = api.IntegratorSettings("mis", 6, True, 3)
    render = api.RenderSettings(64, 48, 6, 4)
    np.testing.assert_array_equal(api.PathTracer(two, settings).render(render)[0],
                                  api.PathTracer(fresh, settings).render(render)[0])


def test_update_mesh_renders_like_a_fresh_build(api):
    doc = sc.job_scene(40_000, 22)
    two = api.Scene(doc.snapshot(), two_level=True)
    k = len(doc.meshes) - 1  # a sphere mesh
    rng = np.random.default_rng(5)
    positions = doc.meshes[k].positions * np.float32(1.1) + rng.normal(0, 0.01, doc.meshes[k].positions.shape)
    positions = positions.astype(np.float32)
    two.update_mesh(k, positions)
    after = sc.SceneDocument(**{f: getattr(doc, f) for f in doc.__dataclass_fields__})
    after.meshes = list(doc.meshes)
    m = doc.meshes[k]
    after.meshes[k] = sc.MeshData(positions, m.corner_positions, m.corner_normals, m.corner_uvs)
    fresh = api.Scene(after.snapshot())
    o, d = rays(after, 100_000, 10)
    assert_same_hits(fresh.intersect(o, d, 0.0, np.inf)[0], two.intersect(o, d, 0.0, np.inf)[0])
    settings = api.IntegratorSettings("mis", 6, True, 3)
    render = api.RenderSettings(64, 48, 6, 4)
    np.testing.assert_array_equal(api.PathTracer(two, settings).render(render)[0],
                                  api.PathTracer(fresh, settings).render(render)[0])


def test_two_level_rejections(api, oracle):
    doc = sc.cornell_box()
    snap = doc.snapshot()
    two = api.Scene(snap, two_level=True)
    flat = api.Scene(snap)
    with pytest.raises(api.MiniRenderError):  # the ceiling light is an area light
        two.update_instances(len(doc.objects) - 1, moved(doc, len(doc.objects) - 1))
    with pytest.raises(api.MiniRenderError):
        flat.update_instances(0, doc)
    with pytest.raises(api.MiniRenderError):
        two.export_bvh()
    with pytest.raises(api.MiniRenderError):
        two.sah_cost()
    with pytest.raises(api.MiniRenderError):
        api.Scene(snap, oracle.OracleScene(snap).export_bvh(), two_level=True)
    with pytest.raises(api.MiniRenderError):
        two.update_mesh(len(doc.meshes) - 1, doc.meshes[-1].positions)  # the light's mesh
