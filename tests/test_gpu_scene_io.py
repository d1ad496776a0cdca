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
