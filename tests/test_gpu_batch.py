"""Batching and serving on the GPU: many jobs in shared waves give each job the image the
single-job render gives (bitwise: same estimator, RNG streams and per-pixel summation order),
whatever it is batched with, however its samples are split into waves, with or without CUDA
graphs; the server admits, pauses, resumes and cancels jobs; a failing job fails alone."""

import time

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


@pytest.fixture(scope="module")
def scenes(api):
    docs = [sc.cornell_box(), sc.job_scene(12_000, 11), sc.job_scene(40_000, 12)]
    return [api.Scene(d.snapshot()) for d in docs]


def job_mix(api, scenes):
    """Uneven jobs: odd sizes, several depths and modes, one over two scenes' worth of rows."""
    R, I = api.RenderSettings, api.IntegratorSettings
    return [
        api.BatchJob(scenes[0], R(64, 48, 5, 1), I("mis", 8, True, 3)),
        api.BatchJob(scenes[1], R(33, 17, 3, 7), I("mis", 4, True, 3)),
        api.BatchJob(scenes[2], R(96, 80, 2, 3), I("bsdf", 12, True, 2)),
        api.BatchJob(scenes[0], R(40, 40, 9, 5), I("light", 6, False, 3)),
        api.BatchJob(scenes[1], R(128, 9, 4, 2), I("mis", 12, True, 3)),
    ]


def plain(api, job):
    tracer = api.PathTracer(job.scene, job.integrator)
    image, _ = tracer.render(job.render)
    return image


@pytest.mark.parametrize("wave_paths,graphs,lanes",
                         [(0, True, 0), (4096, True, 1), (1024, False, 3), (2048, True, 4)])
def test_batch_matches_single_job_renders(api, scenes, wave_paths, graphs, lanes):
    jobs = job_mix(api, scenes)
    images, codes, info = api.render_batch(
        jobs, api.BatchSettings(wave_paths=wave_paths, use_graphs=graphs, concurrent_waves=lanes))
    assert codes == [0] * len(jobs)
    assert info["samples"] == sum(j.render.width * j.render.height * j.render.samples_per_pixel
                                  for j in jobs)
    if wave_paths:
        assert info["waves"] > 1  # small waves split the jobs into frames and row bands
    assert (info["graph_launches"] > 0) == graphs
    for job, image in zip(jobs, images):
        np.testing.assert_array_equal(image, plain(api, job))


def test_unsorted_and_reduced_occupancy_give_same_images(api, scenes):
    jobs = job_mix(api, scenes)[:3]
    ref, _, _ = api.render_batch(jobs)
    other, codes, _ = api.render_batch(
        jobs, api.BatchSettings(wave_paths=8192, trace_blocks_per_sm=2, shade_blocks_per_sm=1,
                                sort_threshold=1 << 30))
    assert codes == [0, 0, 0]
    for a, b in zip(ref, other):
        np.testing.assert_array_equal(a, b)


def test_server_alone_equals_in_mix(api, scenes):
    R, I = api.RenderSettings, api.IntegratorSettings
    probe = (scenes[2], R(72, 56, 6, 9), I("mis", 10, True, 3))
    with api.RenderServer(batch=api.BatchSettings(wave_paths=8192)) as server:
        j = server.submit(*probe)
        assert server.wait(j, 60_000)
        alone = server.result(j)
        assert server.info(j)["state"] == "completed"
    with api.RenderServer(batch=api.BatchSettings(wave_paths=8192)) as server:
        others = [server.submit(s, R(50 + 7 * k, 30 + 5 * k, 2 + k, 100 + k), I("mis", 5 + k, True, 3))
                  for k, s in enumerate(scenes * 2)]
        j = server.submit(*probe)
        others += [server.submit(scenes[k % 3], R(20, 20, 3, 200 + k)) for k in range(4)]
        for job in others + [j]:
            assert server.wait(job, 60_000)
        mixed = server.result(j)
        stats = server.statistics()
        assert stats["completed"] == len(others) + 1
        assert stats["segments"] > stats["waves"]  # jobs shared waves
    np.testing.assert_array_equal(alone, mixed)
    np.testing.assert_array_equal(alone, plain(api, api.BatchJob(*probe)))


def test_server_pause_resume_cancel(api, scenes):
    R = api.RenderSettings
    with api.RenderServer(batch=api.BatchSettings(wave_paths=4096)) as server:
        big = server.submit(scenes[2], R(128, 128, 64, 4))
        victim = server.submit(scenes[1], R(128, 128, 64, 5))
        small = server.submit(scenes[0], R(32, 32, 4, 6))
        assert server.pause(big)
        assert not server.pause(big)  # already paused
        assert server.info(big)["state"] in ("paused", "queued")
        server.cancel(victim)
        assert server.info(victim)["state"] == "cancelled"
        assert server.wait(small, 60_000)
        # Pause acts at the next wave: waves already enqueued with the job still retire. Once
        # they have, the job makes no progress while paused.
        deadline = time.time() + 30
        held = server.info(big)["completed_samples"]
        while True:
            time.sleep(0.2)
            now = server.info(big)["completed_samples"]
            if now == held:
                break
            held = now
            assert time.time() < deadline
        time.sleep(0.3)
        assert server.info(big)["completed_samples"] == held < 128 * 128 * 64
        preview, passes = server.preview(big)
        assert np.isfinite(preview).all() and passes < 64
        assert server.resume(big)
        assert not server.resume(big)
        assert server.wait(big, 120_000)
        assert server.info(big)["state"] == "completed"
        np.testing.assert_array_equal(server.result(big),
                                      plain(api, api.BatchJob(scenes[2], R(128, 128, 64, 4))))
        np.testing.assert_array_equal(server.result(small),
                                      plain(api, api.BatchJob(scenes[0], R(32, 32, 4, 6))))
        with pytest.raises(api.MiniRenderError):
            server.result(victim)
        server.release(small)
        with pytest.raises(api.MiniRenderError):
            server.info(small)
        stats = server.statistics()
        assert stats["cancelled"] == 1 and stats["completed"] == 2


def test_server_budget_queues_jobs(api, scenes):
    R = api.RenderSettings
    one_job = 64 * 64 * 44  # accumulator (32 B) + image (12 B) per pixel
    with api.RenderServer(hbm_budget_bytes=2 * one_job,
                          batch=api.BatchSettings(wave_paths=4096)) as server:
        ids = [server.submit(scenes[k % 3], R(64, 64, 8, k + 1)) for k in range(5)]
        for j in ids:
            assert server.wait(j, 60_000)
        assert all(server.info(j)["state"] == "completed" for j in ids)
        assert server.statistics()["resident_bytes"] == 0
        with pytest.raises(api.MiniRenderError):
            server.submit(scenes[0], R(128, 128, 1, 1))  # alone above the budget


def test_failing_job_fails_alone(api, scenes):
    R, I = api.RenderSettings, api.IntegratorSettings
    doc = sc.cornell_box()
    doc.materials[-1].emission = (3e38, 3e38, 3e38)  # the ceiling light overflows FP32 sums
    hot = api.Scene(doc.snapshot())
    bad = api.BatchJob(hot, R(24, 24, 8, 1), I("mis", 4, True, 3))
    with pytest.raises(api.MiniRenderError) as plain_error:
        plain(api, bad)
    good = job_mix(api, scenes)[:2]
    images, codes, _ = api.render_batch([good[0], bad, good[1]],
                                        api.BatchSettings(wave_paths=4096))
    assert codes[1] == plain_error.value.status
    assert codes[0] == 0 and codes[2] == 0 and images[1] is None
    np.testing.assert_array_equal(images[0], plain(api, good[0]))
    np.testing.assert_array_equal(images[2], plain(api, good[1]))


def test_autotune_returns_a_valid_shape(api, scenes):
    jobs = job_mix(api, scenes)[:2]
    best, rate = api.autotune(jobs)
    assert best.wave_paths in (1 << 21, 1 << 22, 1 << 23) and 1 <= best.concurrent_waves <= 4
    assert rate > 0
    images, codes, _ = api.render_batch(jobs, best)
    assert codes == [0, 0]
    np.testing.assert_array_equal(images[0], plain(api, jobs[0]))


def test_row_bands_assemble_the_frame_bitwise(api, scenes):
    from minirender_b200 import shard
    render = api.RenderSettings(83, 61, 6, 12)
    for scene in scenes[:2]:
        tracer = api.PathTracer(scene, api.IntegratorSettings("mis", 9, True, 3))
        full, stats = tracer.render(render)
        bands = [tracer.render_rows(render, b, e) for b, e in shard.row_bands(render.height, 3)]
        np.testing.assert_array_equal(np.concatenate(bands), full)
        rows, band_stats = tracer.render_rows(render, 0, render.height, statistics=True)
        np.testing.assert_array_equal(rows, full)
        assert band_stats["paths"] == stats["paths"]
    assert tracer.render_rows(render, 5, 5).shape == (0, 83, 3)
    with pytest.raises(api.MiniRenderError):
        tracer.render_rows(render, 10, 62)


def test_repeated_batches_reuse_the_engine_and_report_per_call(api, scenes):
    jobs = job_mix(api, scenes)
    settings = api.BatchSettings(wave_paths=4096, concurrent_waves=2)
    first, codes, a = api.render_batch(jobs, settings)
    second, codes2, b = api.render_batch(jobs, settings)
    assert codes == codes2 == [0] * len(jobs)
    assert a["samples"] == b["samples"] and a["waves"] == b["waves"]  # per-call figures
    assert a["paths"]["paths"] == b["paths"]["paths"]
    for x, y in zip(first, second):
        np.testing.assert_array_equal(x, y)


def test_released_cancelled_job_is_forgotten_safely(api, scenes):
    R = api.RenderSettings
    with api.RenderServer(batch=api.BatchSettings(wave_paths=4096)) as server:
        victim = server.submit(scenes[2], R(128, 128, 32, 8))
        other = server.submit(scenes[1], R(64, 64, 8, 9))
        time.sleep(0.01)
        server.cancel(victim)
        server.release(victim)  # waves carrying it may still be in flight
        with pytest.raises(api.MiniRenderError):
            server.info(victim)
        assert server.wait(other, 60_000)
        np.testing.assert_array_equal(server.result(other),
                                      plain(api, api.BatchJob(scenes[1], R(64, 64, 8, 9))))
