"""The render server under concurrent clients: three threads submit, pause, resume, cancel,
preview and release jobs at random while waves run on two lanes. Every call returns within its
timeout (no deadlock), every job ends completed or cancelled, the counters add up, and every
completed image is bitwise the single-job render's."""

import random
import threading

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


def test_concurrent_clients(api):
    scenes = [api.Scene(sc.cornell_box().snapshot()), api.Scene(sc.job_scene(8_000, 5).snapshot())]
    server = api.RenderServer(batch=api.BatchSettings(wave_paths=4096, concurrent_waves=2))
    outcomes, errors = [], []
    lock = threading.Lock()

    def client(seed):
        rng = random.Random(seed)
        try:
            mine = []
            for k in range(10):
                render = api.RenderSettings(rng.randint(8, 48), rng.randint(8, 48),
                                            rng.randint(1, 8), seed * 100 + k)
                integrator = api.IntegratorSettings("mis", rng.randint(2, 8), True, 3)
                scene = rng.randrange(len(scenes))
                job = server.submit(scenes[scene], render, integrator)
                mine.append((job, scene, render, integrator))
                action = rng.random()
                target = rng.choice(mine)[0]
                if action < 0.2:
                    server.pause(target)
                elif action < 0.4:
                    server.resume(target)
                elif action < 0.5:
                    server.cancel(target)
                elif action < 0.6:
                    server.preview(target)
                server.info(target)
            for job, scene, render, integrator in mine:
                server.resume(job)  # nothing stays paused
            for job, scene, render, integrator in mine:
                assert server.wait(job, 120_000), "job did not finish"
                info = server.info(job)
                assert info["state"] in ("completed", "cancelled"), info
                image = server.result(job) if info["state"] == "completed" else None
                server.release(job)
                with lock:
                    outcomes.append((info["state"], scene, render, integrator, image))
        except Exception as e:  # reported on the main thread
            with lock:
                errors.append(repr(e))

    threads = [threading.Thread(target=client, args=(s,)) for s in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a client is stuck"
    assert not errors, errors
    stats = server.statistics()
    server.close()
    assert len(outcomes) == 30
    assert stats["submitted"] == 30 and stats["completed"] + stats["cancelled"] == 30
    assert stats["completed"] == sum(1 for o in outcomes if o[0] == "completed") > 0
    for state, scene, render, integrator, image in outcomes:
        if state == "completed":
            expected, _ = api.PathTracer(scenes[scene], integrator).render(render)
            np.testing.assert_array_equal(image, expected)


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a
