"""The coherence sort of extension and shadow rays (waves of at least 262,144 paths over scenes of
at least 4,096 triangle slots) reorders the queues only: every path's result, and so every image,
is bit for bit the unsorted render's.

Sorted and unsorted renders of the same jobs are compared: a plain render of a 1M-path frame
(sorted) against a session that advances the frame one sample per pixel per wave (65,536-path
waves, unsorted), and the batched engine with 8M-path waves (sorted) against 128k-path waves
(unsorted), on a job scene with a medium (its vertices take the Morton key) and a two-level
scene (its slots are flat primitive ids).
"""

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


def foggy_room():
    doc = sc.job_scene(40_000, 17)
    doc.media = [sc.MediumRegion((-0.4, 0.0, -0.4), (0.4, 0.6, 0.4), (0.2, 0.3, 0.4),
                                 (0.8, 0.8, 0.8), 0.2)]
    return doc


SCENES = {
    "room": lambda: sc.job_scene(60_000, 3),
    "foggy": foggy_room,
}


@pytest.mark.parametrize("name", list(SCENES))
def test_sorted_render_equals_unsorted_session(api, name):
    doc = SCENES[name]()
    scene = api.Scene(doc.snapshot(), split_references=True)
    assert scene.statistics()["triangles"] >= 4096
    settings = api.IntegratorSettings("mis", 8, True, 3)
    render = api.RenderSettings(256, 256, 16, 4)  # 1,048,576 paths in one wave: sorted
    image, stats = api.PathTracer(scene, settings).render(render)
    session = api.RenderSession()
    session.start(scene, render, settings, api.SessionSettings(0, 16, 1))  # 65,536-path waves
    assert session.wait_for(120000)
    session.wait()
    assert session.progress()["state"] == "completed"
    np.testing.assert_array_equal(session.result(), image)
    session.close()
    assert image.mean() > 0 and stats["shadow_rays"] > 0


def test_sorted_batch_equals_unsorted_batch(api):
    jobs = []
    for seed, two_level in ((5, False), (6, True), (7, False)):
        scene = api.Scene(sc.job_scene(50_000, seed).snapshot(), two_level=two_level)
        jobs.append(api.BatchJob(scene, api.RenderSettings(320, 240, 12, seed),
                                 api.IntegratorSettings("mis", 9, True, 3)))
    sorted_images, codes, _ = api.render_batch(jobs, api.BatchSettings(wave_paths=1 << 23))
    assert codes == [0, 0, 0]
    plain_images, codes, _ = api.render_batch(jobs, api.BatchSettings(wave_paths=1 << 17))
    assert codes == [0, 0, 0]
    for a, b in zip(sorted_images, plain_images):
        np.testing.assert_array_equal(a, b)
