"""A frame larger than one wave (8,388,608 paths) sends its waves round four workspaces, each
with its own stream, so that one wave's last, sparse bounces overlap the next waves' first. The
resolves still accumulate the waves in sample order: the image is bit for bit the single-lane
render's.

A 1024x768 frame at 24 samples per pixel takes three waves of 10, 10 and 4 samples (one lane
each); it is compared with a session that accumulates the same frame two samples per pixel per
wave on one lane. A 1280x720 frame at 40 samples per pixel takes five waves (the first lane takes
a second one); it is compared with five row ranges of one wave each, and its statistics (the sum
of all lanes' counters) with theirs.
"""

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


def test_multi_lane_frame_equals_single_lane_session(api):
    scene = api.Scene(sc.job_scene(60_000, 12).snapshot(), split_references=True)
    settings = api.IntegratorSettings("mis", 8, True, 3)
    render = api.RenderSettings(1024, 768, 24, 5)
    image, stats = api.PathTracer(scene, settings).render(render)
    assert stats["paths"] == 1024 * 768 * 24
    session = api.RenderSession()
    session.start(scene, render, settings, api.SessionSettings(0, 16, 2))
    assert session.wait_for(180000)
    session.wait()
    assert session.progress()["state"] == "completed"
    np.testing.assert_array_equal(session.result(), image)
    session.close()
    assert image.mean() > 0 and stats["shadow_rays"] > 0


def test_five_wave_frame_equals_single_wave_row_ranges(api):
    scene = api.Scene(sc.job_scene(30_000, 4).snapshot())
    tracer = api.PathTracer(scene, api.IntegratorSettings("mis", 6, True, 3))
    render = api.RenderSettings(1280, 720, 40, 8)  # 36,864,000 paths: five waves
    image, stats = tracer.render(render)
    total = dict.fromkeys(("paths", "shadow_rays", "scattering_events", "roulette_terminations"), 0)
    for r0, r1 in ((0, 150), (150, 300), (300, 450), (450, 600), (600, 720)):  # one wave each
        rows, part = tracer.render_rows(render, r0, r1, statistics=True)
        np.testing.assert_array_equal(rows, image[r0:r1])
        for key in total:
            total[key] += part[key]
    for key, value in total.items():
        assert stats[key] == value, key
