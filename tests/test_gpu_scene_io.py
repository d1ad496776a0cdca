"""A scene read from scene JSON v1 + OBJ files renders on the GPU like the oracle renders it
(the image-parity bar of tests/test_gpu_parity.py: per pixel |gpu - cpu| <= 2e-3 max(cpu,
0.05 mean) for at least 99% of pixels, means within 0.5%)."""

import os
import tempfile

import numpy as np
import pytest

from minirender_b200 import scene as sc
from minirender_b200 import scene_io

pytestmark = pytest.mark.gpu


def test_loaded_scene_renders_like_the_oracle(oracle):
    from minirender_b200 import api
    doc = sc.job_scene(6_000, 31)  # a room with displaced spheres of every material
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "room.json")
        scene_io.save_scene(doc, path)
        loaded = scene_io.load_scene(path)
    snap = loaded.snapshot()
    o = oracle.OracleScene(snap, oracle.integrator("mis", 8, True, 3))
    g = api.Scene(snap, o.export_bvh())
    render = api.RenderSettings(64, 48, 8, 2)
    gpu, _ = api.PathTracer(g, api.IntegratorSettings("mis", 8, True, 3)).render(render)
    cpu, _ = o.render(render.c())
    scale = max(float(cpu.mean()), 1e-6)
    ok = np.all(np.abs(gpu - cpu) <= 2e-3 * np.maximum(cpu, 0.05 * scale), axis=2)
    assert ok.mean() >= 0.99, ok.mean()
    assert gpu.mean() == pytest.approx(cpu.mean(), rel=5e-3)


def test_render_command_writes_the_session_image(tmp_path):
    import subprocess
    import sys
    from minirender_b200 import api, image_io
    from tests.test_image_io import read_exr, read_png
    doc = sc.cornell_box()
    scene_path = tmp_path / "cornell.json"
    scene_io.save_scene(doc, str(scene_path))
    out = tmp_path / "renders" / "cornell.png"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    result = subprocess.run([sys.executable, "-m", "minirender_b200.render_cli", "--render",
                             str(scene_path), str(out), "--width", "32", "--height", "24",
                             "--spp", "4", "--seed", "3", "--depth", "6", "--exposure", "0.5"],
                            capture_output=True, text=True, cwd=root, timeout=300)
    assert result.returncode == 0, result.stderr
    assert "EXR and PNG saved." in result.stdout and "paths: 3072" in result.stdout
    exr, _ = read_exr(str(tmp_path / "renders" / "cornell.exr"))
    png = read_png(str(tmp_path / "renders" / "cornell.png"))
    expected, _ = api.PathTracer(scene_io.load_scene(str(scene_path)).snapshot(),
                                 api.IntegratorSettings("mis", 6, True, 3)).render(
        api.RenderSettings(32, 24, 4, 3))
    assert np.array_equal(exr, expected)
    display = api.display_image(expected, 0.5)
    assert np.array_equal(png, image_io.encode_unorm8(image_io.linear_to_srgb(display)))


def test_trace_normals_diagnostic(tmp_path):
    import subprocess
    import sys
    from tests.test_image_io import read_png
    scene_path = tmp_path / "cornell.json"
    scene_io.save_scene(sc.cornell_box(), str(scene_path))
    out = tmp_path / "normals.png"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    result = subprocess.run([sys.executable, "-m", "minirender_b200.render_cli", "--trace-normals",
                             str(scene_path), str(out)], capture_output=True, text=True, cwd=root,
                            timeout=300)
    assert result.returncode == 0, result.stderr
    assert "triangles: 36" in result.stdout and "bounds tests:" in result.stdout
    image = read_png(str(out))
    assert image.shape == (256, 256, 3)
    # The centre of the image looks at the back wall or a box: a hit with a unit normal.
    from minirender_b200 import image_io
    centre = image[128, 128].astype(int)
    assert centre.sum() > 0
    # The floor near the bottom centre faces +y: normal (0, 1, 0) -> (0.5, 1, 0.5).
    expected = image_io.encode_unorm8(image_io.linear_to_srgb(np.array([0.5, 1.0, 0.5], np.float32)))
    assert np.abs(image[250, 128].astype(int) - expected.astype(int)).max() <= 1
