"""The integration guide's SceneSnapshot binding, compiled against the reference's own headers.

INTEGRATION.md's C++ block (the `to_b200` conversion and the lines that replace render_cli.cpp's
session) is extracted verbatim and compiled with g++ against the reference's
include/minirender/scene/scene.hpp, render/path_tracer.hpp and render/render_session.hpp, using
the project's GLM stand-in (tests/binding/glm), and linked against this library and the oracle.
The program (tests/binding/snapshot_binding.cpp) converts a snapshot with two meshes, three
instances (a textured, normal-mapped floor, a conductor, an emitter), a directional light, a
medium and an environment map, and renders it with the oracle; the same scene built through the
Python scene model must render bitwise identically. Runs where MINIRENDER_REFERENCE_INCLUDE names
the reference's include/ directory (the reference is not shipped with this repository).
"""

import os
import re
import subprocess

import numpy as np
import pytest

from minirender_b200 import _abi
from minirender_b200 import scene as sc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE_INCLUDE = os.environ.get("MINIRENDER_REFERENCE_INCLUDE", "")
F32 = np.float32

pytestmark = pytest.mark.skipif(
    not REFERENCE_INCLUDE or not os.path.isdir(os.path.join(REFERENCE_INCLUDE, "minirender")),
    reason="MINIRENDER_REFERENCE_INCLUDE does not name the reference's include/ directory")


def guide_blocks():
    """The guide's C++ block split at the render_cli comment: (declarations, session lines)."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.search(r"```cpp\n(.*?)```", text, re.S).group(1)
    head, tail = block.split("// render_cli.cpp", 1)
    tail = tail.split("\n", 1)[1]  # drop the rest of the comment line
    return head, tail


def texture(w, h, seed):
    """snapshot_binding.cpp's texture() in the same FP32 operations."""
    y, x = np.mgrid[0:h, 0:w]
    v = ((x * 7 + y * 13) % 11).astype(F32) / F32(10)
    rgb = np.stack([F32(0.2) + F32(0.6) * v,
                    np.full_like(v, F32(0.5) + F32(0.25) * F32(seed)),
                    F32(0.9) - F32(0.5) * v], axis=2)
    return sc.TextureData(rgb.astype(F32))


def quad(down):
    positions = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F32)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], F32)
    tris = np.array([[0, 3, 2], [0, 2, 1]], np.uint32)
    if down:
        tris = tris[:, ::-1].copy()
    normals = np.zeros((2, 3, 3), F32)
    normals[..., 1] = -1 if down else 1
    return sc.MeshData(positions, tris, normals, uv[tris])


def python_scene():
    doc = sc.SceneDocument()
    doc.camera = sc.Camera((0.3, 2.5, 3.0), (0.0, 0.2, 0.0), (0.0, 1.0, 0.0), 50.0, 0.05, 100.0)
    doc.environment = (0.05, 0.06, 0.08)
    doc.textures = [texture(4, 4, 0.0), texture(2, 2, 0.5), texture(8, 4, 1.0)]
    doc.environment_texture = 2
    doc.environment_strength = 0.75
    doc.environment_rotation_degrees = 30.0
    doc.meshes = [quad(False), quad(True)]
    doc.materials = [
        sc.Material("diffuse", (0.9, 0.8, 0.7), base_color_texture=0, texture_filter="bilinear",
                    normal_texture=1, normal_scale=0.6),
        sc.Material("conductor", (0.95, 0.7, 0.4), roughness=0.3),
        sc.Material("diffuse", (0.0, 0.0, 0.0), (6.0, 5.0, 4.0), double_sided=False),
    ]
    doc.objects = [
        sc.SceneObject(0, 0, sc.Transform((0, 0, 0), (0, 0, 0), (3, 1, 3))),
        sc.SceneObject(0, 1, sc.Transform((0.5, 0.4, -0.5), (0, 0, 0), (0.5, 1.0, 0.25))),
        sc.SceneObject(1, 2, sc.Transform((-0.5, 2.0, 0.5), (0, 0, 0), (0.4, 1.0, 0.4))),
    ]
    doc.directional_lights = [sc.DirectionalLight((-1.0, -3.0, -0.5), (1.0, 0.9, 0.8), 2.0)]
    doc.media = [sc.MediumRegion((-2.0, 0.0, -2.0), (2.0, 1.5, 2.0), (0.02, 0.03, 0.04),
                                 (0.1, 0.1, 0.1), 0.3)]
    return doc


def test_guide_binding_compiles_against_reference_headers_and_converts(tmp_path, oracle):
    head, tail = guide_blocks()
    (tmp_path / "to_b200.inc").write_text(head)
    (tmp_path / "render_cli.inc").write_text(tail)
    _abi.load_library()  # the in-tree library is built
    lib_dir = os.path.dirname(_abi.LIBRARY_PATH)
    oracle_dir = os.path.join(ROOT, "oracle", "_build")
    exe = tmp_path / "binding"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Werror=narrowing",
           "-I", str(tmp_path), "-I", os.path.join(ROOT, "tests", "binding"),
           "-I", REFERENCE_INCLUDE, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "binding", "snapshot_binding.cpp"), "-o", str(exe),
           "-L", lib_dir, "-lminirender_b200", f"-Wl,-rpath,{lib_dir}",
           "-L", oracle_dir, "-loracle", f"-Wl,-rpath,{oracle_dir}"]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-4000:]
    out = tmp_path / "image.f32"
    run = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr + run.stdout
    converted = np.fromfile(out, F32).reshape(16, 24, 3)

    o = oracle.OracleScene(python_scene().snapshot(), oracle.integrator("mis", 5, True, 3))
    expected, _ = o.render(_abi.RenderSettings(24, 16, 4, 7), threads=1)
    assert np.isfinite(converted).all() and converted.mean() > 0
    np.testing.assert_array_equal(converted, expected)
