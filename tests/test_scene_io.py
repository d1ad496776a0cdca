"""Scene JSON v1 and OBJ ingestion (src/assets/scene_io.cpp:45-160, src/assets/obj_loader.cpp):
keys, defaults, id references, quad triangulation along the shorter diagonal, corner normals and
the reference's rejections; generated scenes round-trip; the reference's own scene files load
(when MINIRENDER_REFERENCE_SCENES names its scenes/ folder) and the oracle renders one; the
fixtures of two of them (tests/golden/scenes) load and render."""

import json
import os
import tempfile

import numpy as np
import pytest

from minirender_b200 import scene as sc
from minirender_b200 import scene_io

# The reference checkout's scenes/ folder, when the environment names it (the reference tree is
# not shipped with this repository); the test that loads every reference scene skips otherwise.
# tests/golden/scenes holds fixtures of two of them for the tests that must always run.
REFERENCE_SCENES = os.environ.get("MINIRENDER_REFERENCE_SCENES", "")


def write(directory, name, text):
    path = os.path.join(directory, name)
    with open(path, "w") as f:
        f.write(text)
    return path


def test_obj_corners_normals_and_triangulation():
    with tempfile.TemporaryDirectory() as d:
        path = write(d, "m.obj", "\n".join([
            "# quad whose 0-2 diagonal is shorter, a quad whose 1-3 diagonal is, a triangle",
            "v 0 0 0", "v 2 0 0", "v 2.5 1 0", "v 0.5 1 0",      # 0-2 longer than 1-3
            "v 0 0 1", "v 1 0 1", "v 1 3 1", "v 0 1 1",          # 0-2 longer too; see below
            "vn 0 0 2", "vt 0.25 0.5",
            "o shape", "g group", "s 1", "usemtl anything",
            "f 1 2 3 4",
            "f 5/1 6/1 7/1 8/1",
            "f -3//1 -2//1 -1//1",
        ]))
        mesh = scene_io.load_obj(path)
    p = mesh.positions
    assert p.shape == (8, 3) and mesh.triangle_count == 5
    d02 = np.sum((p[2] - p[0]) ** 2); d13 = np.sum((p[3] - p[1]) ** 2)
    expected = [[0, 1, 2], [0, 2, 3]] if d02 < d13 else [[0, 1, 3], [1, 2, 3]]
    assert mesh.corner_positions[:2].tolist() == expected
    d02 = np.sum((p[6] - p[4]) ** 2); d13 = np.sum((p[7] - p[5]) ** 2)
    expected = [[4, 5, 6], [4, 6, 7]] if d02 < d13 else [[4, 5, 7], [5, 6, 7]]
    assert mesh.corner_positions[2:4].tolist() == expected
    assert mesh.corner_positions[4].tolist() == [5, 6, 7]  # relative indices
    assert np.allclose(mesh.corner_normals[4], [0, 0, 1])  # vn normalised
    assert np.allclose(mesh.corner_normals[0], [0, 0, 1])  # geometric normal without vn
    assert np.allclose(mesh.corner_uvs[2], [[0.25, 0.5]] * 3)
    assert np.allclose(mesh.corner_uvs[0], 0)


@pytest.mark.parametrize("body,message", [
    ("v 0 0 0\nv 1 0 0\nv 2 0 0\nf 1 2 3\n", "degenerate"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", "vertex index"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 0\nf 1//1 2//1 3//1\n", "normal is zero"),
])
def test_obj_rejections(body, message):
    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(ValueError, match=message):
            scene_io.load_obj(write(d, "bad.obj", body))


def minimal_scene(**overrides):
    data = {
        "version": 1,
        "camera": {"position": [0, 1, 3], "target": [0, 1, 0], "up": [0, 1, 0],
                   "vertical_fov": 40, "near": 0.05, "far": 50},
        "environment": [0.1, 0.2, 0.3],
        "materials": [{"id": "white", "kind": "diffuse", "base_color": [0.7, 0.7, 0.7]},
                      {"id": "lamp", "kind": "diffuse", "base_color": [0, 0, 0],
                       "emission": [5, 5, 5], "double_sided": False}],
        "meshes": [{"id": "plane", "source": "plane.obj"}],
        "objects": [{"id": "floor", "mesh": "plane", "material": "white",
                     "transform": {"translation": [0, 0, 0], "rotation": [0, 0, 0],
                                   "scale": [1, 1, 1]}},
                    {"id": "light", "mesh": "plane", "material": "lamp", "visible": True,
                     "transform": {"translation": [0, 2, 0], "rotation": [180, 0, 0],
                                   "scale": [0.2, 1, 0.2]}}],
        "directional_lights": [{"id": "sun", "direction": [0, -1, 0], "color": [1, 1, 1],
                                "intensity": 2}],
    }
    data.update(overrides)
    return data


PLANE = "v -1 0 -1\nv -1 0 1\nv 1 0 1\nv 1 0 -1\nf 1 2 3 4\n"


def test_scene_keys_defaults_and_references():
    with tempfile.TemporaryDirectory() as d:
        write(d, "plane.obj", PLANE)
        data = minimal_scene(media=[{"id": "fog", "minimum": [-1, 0, -1], "maximum": [1, 2, 1],
                                     "absorption": [0.1, 0.2, 0.3], "scattering": [0.4, 0.4, 0.4],
                                     "anisotropy": 0.25}])
        doc = scene_io.load_scene(write(d, "s.json", json.dumps(data)))
    assert doc.camera.aperture_radius == 0.0 and doc.camera.focus_distance == 4.0
    assert doc.materials[0].roughness == pytest.approx(0.35) and doc.materials[0].ior == 1.5
    assert doc.materials[0].double_sided and not doc.materials[1].double_sided
    assert doc.materials[0].emission == (0.0, 0.0, 0.0)
    assert [o.mesh for o in doc.objects] == [0, 0] and [o.material for o in doc.objects] == [0, 1]
    assert doc.media[0].enabled and doc.media[0].anisotropy == 0.25
    assert doc.directional_lights[0].intensity == 2.0
    assert doc.snapshot().triangle_count == 4


@pytest.mark.parametrize("change,message", [
    ({"version": 2}, "version"),
    ({"objects": [{"id": "x", "mesh": "nope", "material": "white",
                   "transform": {"translation": [0, 0, 0], "rotation": [0, 0, 0],
                                 "scale": [1, 1, 1]}}]}, "missing mesh"),
    ({"materials": [{"id": "white", "kind": "plastic", "base_color": [1, 1, 1]}]}, "kind"),
    ({"materials": [{"id": "white", "kind": "diffuse", "base_color": [1, 1, 1],
                     "base_color_texture": "wood"}]}, "missing texture: wood"),
    ({"environment_map": {"texture": "sky"}}, "Environment references missing texture: sky"),
    ({"materials": [{"id": "white", "kind": "diffuse", "base_color": [1, 1, 1],
                     "texture_filter": "cubic"}]}, "texture filter"),
    ({"textures": [{"id": "t", "source": "t.png", "encoding": "gamma"}]}, "encoding"),
    ({"camera": {"position": [0, 1, 3]}}, "missing key"),
])
def test_scene_rejections(change, message):
    with tempfile.TemporaryDirectory() as d:
        write(d, "plane.obj", PLANE)
        with pytest.raises(ValueError, match=message):
            scene_io.load_scene(write(d, "s.json", json.dumps(minimal_scene(**change))))


def test_generated_scene_round_trips(oracle):
    doc = sc.cornell_box()
    doc.media = [sc.MediumRegion((-0.5, 0, -0.5), (0.5, 1, 0.5), (0.1, 0.1, 0.1), (0.3, 0.3, 0.3), 0.2)]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "cornell.json")
        scene_io.save_scene(doc, path)
        back = scene_io.load_scene(path)
    a, b = doc.snapshot(), back.snapshot()
    assert np.array_equal(a.world_triangles(), b.world_triangles())
    from minirender_b200 import _abi
    render = _abi.RenderSettings(12, 9, 2, 4)
    settings = oracle.integrator("mis", 4, True, 3)
    ia, _ = oracle.OracleScene(a, settings).render(render, threads=2)
    ib, _ = oracle.OracleScene(b, settings).render(render, threads=2)
    assert np.array_equal(ia, ib)


@pytest.mark.skipif(not REFERENCE_SCENES or not os.path.isdir(REFERENCE_SCENES),
                    reason="MINIRENDER_REFERENCE_SCENES does not name the reference's scenes/")
def test_reference_scene_files_load(oracle):
    loaded = 0
    for name in sorted(os.listdir(REFERENCE_SCENES)):
        if not name.endswith(".json") or name == "resource_catalog.json":
            continue
        path = os.path.join(REFERENCE_SCENES, name)
        doc = scene_io.load_scene(path)
        assert doc.snapshot().triangle_count > 0
        loaded += 1
    assert loaded >= 21  # every scene file the reference ships, the two textured ones included
    from minirender_b200 import _abi
    doc = scene_io.load_scene(os.path.join(REFERENCE_SCENES, "cornell-box.json"))
    image, stats = oracle.OracleScene(doc.snapshot(), oracle.integrator("mis", 4, True, 3)).render(
        _abi.RenderSettings(16, 12, 2, 1), threads=2)
    assert np.isfinite(image).all() and image.mean() > 0 and stats["paths"] == 16 * 12 * 2


def test_reference_scene_fixtures_load_and_render(oracle):
    from minirender_b200 import _abi
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes")
    for name, triangles in (("studio", 26), ("path-room", 36)):
        doc = scene_io.load_scene(os.path.join(golden, f"{name}.json"))
        assert doc.snapshot().triangle_count == triangles
        image, stats = oracle.OracleScene(doc.snapshot(), oracle.integrator("mis", 4, True, 3)).render(
            _abi.RenderSettings(16, 12, 2, 1), threads=2)
        assert np.isfinite(image).all() and image.mean() > 0 and stats["paths"] == 16 * 12 * 2


def write_png_rgb(path, rgb8):
    """An 8-bit RGB PNG of (h, w, 3) uint8 samples."""
    import struct
    import zlib
    h, w = rgb8.shape[:2]
    raw = b"".join(b"\x00" + row.tobytes() for row in rgb8.reshape(h, w * 3))

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body))

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0))
                + chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))


def test_textures_load_decode_and_round_trip():
    from minirender_b200 import image_io
    rng = np.random.default_rng(3)
    rgb8 = rng.integers(0, 256, (5, 7, 3)).astype(np.uint8)
    with tempfile.TemporaryDirectory() as d:
        write(d, "plane.obj", PLANE)
        write_png_rgb(os.path.join(d, "albedo.png"), rgb8)
        write_png_rgb(os.path.join(d, "normals.png"), rgb8)
        image_io.write_exr(os.path.join(d, "sky.exr"), rng.uniform(0, 4, (8, 16, 3)).astype(np.float32))
        data = minimal_scene(
            textures=[{"id": "albedo", "source": "albedo.png"},
                      {"id": "normals", "source": "normals.png", "encoding": "linear"},
                      {"id": "sky", "source": "sky.exr", "encoding": "linear"}],
            environment_map={"texture": "sky", "strength": 2.0, "rotation_degrees": 30.0})
        data["materials"][0].update({"base_color_texture": "albedo", "normal_texture": "normals",
                                     "normal_scale": 0.5, "normal_flip_y": True,
                                     "texture_filter": "bilinear"})
        doc = scene_io.load_scene(write(d, "s.json", json.dumps(data)))
        # sRGB 8-bit samples decode through srgb_to_linear, linear ones scale by 1/255
        expected = image_io.srgb_to_linear(rgb8.astype(np.float32) / np.float32(255))
        np.testing.assert_array_equal(doc.textures[0].rgb, expected)
        np.testing.assert_array_equal(doc.textures[1].rgb, rgb8.astype(np.float32) / np.float32(255))
        m = doc.materials[0]
        assert (m.base_color_texture, m.normal_texture, m.texture_filter) == (0, 1, "bilinear")
        assert m.normal_scale == 0.5 and m.normal_flip_y
        assert (doc.environment_texture, doc.environment_strength,
                doc.environment_rotation_degrees) == (2, 2.0, 30.0)
        saved = os.path.join(d, "saved", "copy.json")
        os.makedirs(os.path.dirname(saved))
        scene_io.save_scene(doc, saved)
        back = scene_io.load_scene(saved)
        for a, b in zip(doc.textures, back.textures):
            np.testing.assert_array_equal(a.rgb, b.rgb)
        assert back.materials[0] == doc.materials[0] and back.environment_texture == 2
        # a normal map must be linear; EXR textures must be declared linear
        data["materials"][0]["normal_texture"] = "albedo"
        with pytest.raises(ValueError, match="linear texture"):
            scene_io.load_scene(write(d, "s2.json", json.dumps(data)))
        data["materials"][0]["normal_texture"] = "normals"
        data["textures"][2]["encoding"] = "srgb"
        with pytest.raises(ValueError, match="EXR textures require linear"):
            scene_io.load_scene(write(d, "s3.json", json.dumps(data)))
