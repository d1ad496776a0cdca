"""Textures, normal maps and the environment map in the oracle, against closed forms:

  * base-colour textures (Texture::sample at lod 0, src/core/texture.cpp:100-139): a floor under
    a directional light straight above returns base_color x texture(uv) x E / pi from a single
    light-sampled path, with the texture restated here in FP32 (nearest and bilinear, Repeat
    addressing, the image's origin at the top left);
  * a flat normal map (every texel (0.5, 0.5, 1)) leaves shading unchanged, a tilted one does not
    (SceneBvh::surface_hit's normal-map step, src/render/bvh.cpp:334-358);
  * the environment map (EnvironmentLight, src/render/light.cpp:61-195): rays that escape return
    the constant plus strength x the bilinear lat-long lookup restated here in FP64; a map of one
    constant value behaves as a constant environment for every sampling mode (its importance
    density is exactly uniform); with a bright patch, BSDF, light and MIS estimates agree (the
    sampling density and the pdf used for MIS are consistent) and MIS has the lowest variance.
"""

import math

import numpy as np
import pytest

from minirender_b200 import scene as sc
from tests.test_oracle_golden import floor_doc

F32 = np.float32


def texture_fp32(tex, u, v, filter_="bilinear"):
    """Texture::sample at lod 0 in FP32 (texture.cpp:17-22, 100-139)."""
    h, w = tex.shape[:2]
    u, v = F32(u), F32(v)
    cx = F32(u - np.floor(u))
    cy = F32(F32(1) - F32(v - np.floor(v)))
    if filter_ == "nearest":
        x = int(np.floor(F32(cx * F32(w))))
        y = int(np.floor(F32(cy * F32(h))))
        return tex[y % h, x % w].astype(np.float64)
    x = F32(F32(cx * F32(w)) - F32(0.5))
    y = F32(F32(cy * F32(h)) - F32(0.5))
    ix, iy = int(np.floor(x)), int(np.floor(y))
    tx, ty = F32(x - np.floor(x)), F32(y - np.floor(y))

    def mix(a, b, t):
        return (a * F32(F32(1) - t)).astype(F32) + (b * t).astype(F32)

    def texel(px, py):
        return tex[py % h, px % w]
    return mix(mix(texel(ix, iy), texel(ix + 1, iy), tx),
               mix(texel(ix, iy + 1), texel(ix + 1, iy + 1), tx), ty).astype(np.float64)


def lit_floor(texture, filter_="bilinear"):
    doc = floor_doc("diffuse", 0.6)
    doc.environment = (0.0, 0.0, 0.0)
    doc.textures = [sc.TextureData(texture)]
    doc.materials[0].base_color_texture = 0
    doc.materials[0].texture_filter = filter_
    irradiance = float(F32(math.pi))
    doc.directional_lights.append(sc.DirectionalLight((0, -1, 0), (1, 1, 1), irradiance))
    return doc, irradiance


def floor_uv(x, z):
    """The floor quad's UVs at world (x, 0, z): the quad spans [-4, 4]^2 with u along z, v along x."""
    return (z / 4 + 1) / 2, (x / 4 + 1) / 2


@pytest.mark.parametrize("filter_", ["nearest", "bilinear", "trilinear"])
def test_base_colour_texture_under_a_directional_light(oracle, filter_):
    rng = np.random.default_rng(7)
    texture = rng.uniform(0.05, 1.0, (5, 7, 3)).astype(F32)
    doc, irradiance = lit_floor(texture, filter_)
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator("light", 1, False, 3))
    xs, zs = np.meshgrid(np.linspace(-3.7, 3.6, 9), np.linspace(-3.55, 3.85, 8))
    origins = np.stack([xs.ravel(), np.ones(xs.size), zs.ravel()], 1)
    keys = np.zeros((len(origins), 3), np.uint64)
    keys[:, 2] = np.arange(len(origins))
    rad, _ = o.trace_paths(origins, [[0, -1, 0]] * len(origins), 0, 100, keys)
    for i, (x, z) in enumerate(zip(xs.ravel(), zs.ravel())):
        u, v = floor_uv(x, z)
        # trilinear at lod 0 is the level-0 bilinear value
        tex = texture_fp32(texture, u, v, "nearest" if filter_ == "nearest" else "bilinear")
        expected = F32(0.6).astype(np.float64) * tex * irradiance / math.pi
        np.testing.assert_allclose(rad[i], expected, rtol=2e-6, atol=1e-9)


def test_flat_normal_map_keeps_shading_and_a_tilted_one_changes_it(oracle):
    from minirender_b200 import _abi
    base = sc.job_scene(3_000, 4)
    render = _abi.RenderSettings(24, 18, 4, 3)
    settings = oracle.integrator("mis", 4, True, 3)
    plain, _ = oracle.OracleScene(base.snapshot(), settings).render(render, threads=2)
    for value, same in (((0.5, 0.5, 1.0), True), ((0.9, 0.5, 0.6), False)):
        doc = sc.job_scene(3_000, 4)
        doc.textures = [sc.TextureData(np.broadcast_to(F32(value), (2, 2, 3)).copy())]
        for m in doc.materials:
            m.normal_texture = 0
        mapped, _ = oracle.OracleScene(doc.snapshot(), settings).render(render, threads=2)
        if same:
            np.testing.assert_allclose(mapped, plain, rtol=1e-5, atol=1e-7)
        else:
            assert np.abs(mapped - plain).max() > 1e-3


def environment_fp64(env, constant, strength, rotation_degrees, d):
    """EnvironmentLight::evaluate in FP64 (light.cpp:112-143)."""
    h, w = env.shape[:2]
    d = np.asarray(d, np.float64)
    d = d / np.sqrt(d @ d)
    rotation = math.remainder(rotation_degrees, 360.0) * math.pi / 180
    u = (math.atan2(d[2], d[0]) + rotation) / (2 * math.pi)
    u -= math.floor(u)
    v = math.atan2(math.hypot(d[0], d[2]), d[1]) / math.pi
    x, y = u * w - 0.5, v * h - 0.5
    ix, iy = math.floor(x), math.floor(y)
    tx, ty = x - ix, y - iy

    def texel(c, r):
        return np.maximum(env[min(max(r, 0), h - 1), c % w].astype(np.float64), 0)

    def mix(a, b, t):
        return a * (1 - t) + b * t
    value = mix(mix(texel(ix, iy), texel(ix + 1, iy), tx), mix(texel(ix, iy + 1), texel(ix + 1, iy + 1), tx), ty)
    return np.asarray(constant, F32).astype(np.float64) + strength * value


def sky_scene(env, strength=1.5, rotation=30.0, constant=(0.1, 0.2, 0.3)):
    doc = floor_doc("diffuse", 0.6)
    doc.environment = constant
    doc.textures = [sc.TextureData(env)]
    doc.environment_texture = 0
    doc.environment_strength = strength
    doc.environment_rotation_degrees = rotation
    return doc


def test_escaping_rays_see_the_environment_map(oracle):
    rng = np.random.default_rng(11)
    env = rng.uniform(-0.2, 3.0, (9, 16, 3)).astype(F32)  # negative texels count as 0
    doc = sky_scene(env)
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator("mis", 3, False, 3))
    dirs = rng.normal(size=(200, 3))
    dirs[:, 1] = np.abs(dirs[:, 1]) + 0.05  # upwards, away from the floor below the origin
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    keys = np.zeros((200, 3), np.uint64)
    rad, _ = o.trace_paths([[0, 1, 0]] * 200, dirs, 0, 1e4, keys)
    for i in range(200):
        expected = environment_fp64(env, (0.1, 0.2, 0.3), 1.5, 30.0, dirs[i])
        np.testing.assert_allclose(rad[i], expected, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("mode", ["bsdf", "light", "mis"])
def test_uniform_map_behaves_as_a_constant_environment(oracle, mode):
    from tests.test_oracle_golden import estimate
    doc = sky_scene(np.full((8, 16, 3), 0.5, F32), strength=1.5, rotation=10.0, constant=(0.25, 0.25, 0.25))
    o = oracle.OracleScene(doc.snapshot(), oracle.integrator(mode, 1, False, 3))
    mean, se, _ = estimate(o, 8192, 81)
    assert abs(mean - float(F32(0.6))) < 5 * se + 1e-9


def test_importance_sampled_map_estimators_agree(oracle):
    from tests.test_oracle_golden import estimate
    env = np.full((32, 64, 3), 0.05, F32)
    env[4:8, 10:16] = 40.0  # a bright patch high in the sky
    doc = sky_scene(env, strength=1.0, rotation=-45.0, constant=(0.0, 0.0, 0.0))
    means = {}
    for mode in ("bsdf", "light", "mis"):
        o = oracle.OracleScene(doc.snapshot(), oracle.integrator(mode, 1, False, 3))
        means[mode] = estimate(o, 60000, 5)[:2]
    reference, ref_se = means["mis"]
    for mode in ("bsdf", "light"):
        mean, se = means[mode]
        assert abs(mean - reference) < 5 * math.hypot(se, ref_se), (mode, means)
    # MIS combines the map's importance sampling with BSDF sampling: lower variance than either
    # (light sampling alone keeps fireflies where bilinear lookup bleeds the patch into
    # low-density texels, the reason the reference mixes in uniform density).
    assert means["mis"][1] < 0.5 * min(means["light"][1], means["bsdf"][1])
