"""Textures, normal maps and the environment map on the GPU (through the C ABI), against closed
forms and the FP64 oracle (the oracle's own texture tests are tests/test_oracle_textures.py):

  * a textured floor under a directional light straight above returns base_color x texture(uv) x
    E / pi (the texture restated in FP32 here) within 1e-5 relative;
  * escaping rays return the environment constant plus strength x the lat-long lookup (FP64
    restatement) within 2e-5 relative;
  * a map of one constant value behaves as a constant environment in every sampling mode (5 sigma);
  * images at equal seeds: a room with a textured floor, normal-mapped spheres and an
    importance-sampled environment map, and the reference's own `studio-textured` scene, against
    the oracle with the image-parity bar of tests/test_gpu_parity.py (per pixel |gpu - cpu| <=
    2e-3 x max(cpu, 0.05 mean) for at least 99% of pixels, means within 0.5%);
  * a two-level scene with textures renders bitwise like the flattened one.
"""

import math
import os

import numpy as np
import pytest

from minirender_b200 import scene as sc
from minirender_b200 import scene_io
from tests.test_oracle_textures import (F32, environment_fp64, floor_uv, lit_floor, sky_scene,
                                        texture_fp32)

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes")


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


@pytest.mark.parametrize("filter_", ["nearest", "bilinear", "trilinear"])
def test_base_colour_texture_under_a_directional_light(api, filter_):
    rng = np.random.default_rng(7)
    texture = rng.uniform(0.05, 1.0, (5, 7, 3)).astype(F32)
    doc, irradiance = lit_floor(texture, filter_)
    tracer = api.PathTracer(doc.snapshot(), api.IntegratorSettings("light", 1, False, 3))
    xs, zs = np.meshgrid(np.linspace(-3.7, 3.6, 9), np.linspace(-3.55, 3.85, 8))
    origins = np.stack([xs.ravel(), np.ones(xs.size), zs.ravel()], 1)
    keys = np.zeros((len(origins), 3), np.uint64)
    keys[:, 2] = np.arange(len(origins))
    rad, _ = tracer.trace(origins, [[0, -1, 0]] * len(origins), 0, 100, keys)
    for i, (x, z) in enumerate(zip(xs.ravel(), zs.ravel())):
        u, v = floor_uv(x, z)
        tex = texture_fp32(texture, u, v, "nearest" if filter_ == "nearest" else "bilinear")
        expected = 0.6 * tex * irradiance / math.pi
        np.testing.assert_allclose(rad[i], expected, rtol=1e-5, atol=1e-7)


def test_escaping_rays_see_the_environment_map(api):
    rng = np.random.default_rng(11)
    env = rng.uniform(-0.2, 3.0, (9, 16, 3)).astype(F32)
    tracer = api.PathTracer(sky_scene(env).snapshot(), api.IntegratorSettings("mis", 3, False, 3))
    dirs = rng.normal(size=(400, 3))
    dirs[:, 1] = np.abs(dirs[:, 1]) + 0.05
    dirs = (dirs / np.linalg.norm(dirs, axis=1, keepdims=True)).astype(F32)
    keys = np.zeros((400, 3), np.uint64)
    rad, _ = tracer.trace([[0, 1, 0]] * 400, dirs, 0, 1e4, keys)
    for i in range(400):
        expected = environment_fp64(env, (0.1, 0.2, 0.3), 1.5, 30.0, dirs[i])
        np.testing.assert_allclose(rad[i], expected, rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("mode", ["bsdf", "light", "mis"])
def test_uniform_map_behaves_as_a_constant_environment(api, mode):
    from tests.test_gpu_parity import estimate
    doc = sky_scene(np.full((8, 16, 3), 0.5, F32), strength=1.5, rotation=10.0,
                    constant=(0.25, 0.25, 0.25))
    mean, se, _ = estimate(api.PathTracer(doc.snapshot(), api.IntegratorSettings(mode, 1, False, 3)),
                           8192, 81)
    assert abs(mean - 0.6) < 5 * se + 2e-6


def textured_room():
    """A room with a checker-textured floor (sRGB-like values), normal-mapped spheres and an
    environment map with a bright patch seen through the open front."""
    doc = sc.job_scene(6_000, 31)
    rng = np.random.default_rng(5)
    checker = np.kron((np.indices((8, 8)).sum(0) % 2).astype(F32)[..., None] * F32(0.7) + F32(0.2),
                      np.ones((4, 4, 1), F32))
    checker = np.repeat(checker, 3, axis=2).astype(F32)
    bumps = np.stack([0.5 + 0.3 * np.sin(np.arange(16) / 2.0)[None, :].repeat(16, 0),
                      0.5 + 0.3 * np.cos(np.arange(16) / 3.0)[:, None].repeat(16, 1),
                      np.full((16, 16), 0.8)], axis=2).astype(F32)
    sky = np.full((16, 32, 3), 0.2, F32)
    sky[3:6, 5:9] = 12.0
    doc.textures = [sc.TextureData(checker), sc.TextureData(bumps), sc.TextureData(sky)]
    doc.materials[0].base_color_texture = 0  # the white walls, floor included
    doc.materials[0].texture_filter = "bilinear"
    for m in doc.materials[5:]:               # the spheres
        m.normal_texture = 1
        m.normal_scale = 0.7
    doc.environment_texture = 2
    doc.environment_strength = 1.0
    doc.environment_rotation_degrees = 20.0
    doc.environment = (0.05, 0.05, 0.05)
    return doc


def image_parity(api, oracle, doc, render, settings_args):
    snap = doc.snapshot()
    o = oracle.OracleScene(snap, oracle.integrator(*settings_args))
    g = api.Scene(snap, o.export_bvh())
    gpu, gstats = api.PathTracer(g, api.IntegratorSettings(*settings_args)).render(render)
    cpu, cstats = o.render(render.c())
    scale = max(float(cpu.mean()), 1e-6)
    ok = np.all(np.abs(gpu - cpu) <= 2e-3 * np.maximum(cpu, 0.05 * scale), axis=2)
    print(f"pixels within tolerance {ok.mean():.4f}, means {gpu.mean():.5f} vs {cpu.mean():.5f}")
    assert ok.mean() >= 0.99, ok.mean()
    assert gpu.mean() == pytest.approx(cpu.mean(), rel=5e-3)
    assert gstats["shadow_rays"] == pytest.approx(cstats["shadow_rays"], rel=2e-3)
    return gpu


def test_textured_room_matches_oracle(api, oracle):
    image_parity(api, oracle, textured_room(), api.RenderSettings(96, 72, 8, 3), ("mis", 6, True, 3))


def test_reference_textured_studio_matches_oracle(api, oracle):
    doc = scene_io.load_scene(os.path.join(GOLDEN, "studio-textured.json"))
    assert doc.textures and any(m.base_color_texture is not None for m in doc.materials)
    image_parity(api, oracle, doc, api.RenderSettings(96, 72, 8, 9), ("mis", 8, True, 3))


def test_two_level_textured_scene_equals_flattened(api):
    doc = textured_room()
    settings = api.IntegratorSettings("mis", 6, True, 3)
    render = api.RenderSettings(64, 48, 6, 2)
    a, _ = api.PathTracer(api.Scene(doc.snapshot()), settings).render(render)
    b, _ = api.PathTracer(api.Scene(doc.snapshot(), two_level=True), settings).render(render)
    np.testing.assert_array_equal(a, b)
