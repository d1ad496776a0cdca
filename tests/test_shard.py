"""Sharding over ranks: row bands and job shares cover the work exactly once, and the gather on
rank 0 reassembles the one-process result bit for bit. The distributed cases run two gloo ranks
on the CPU with the oracle standing in for each rank's GPU renderer (the GPU's own row-band
entry point is checked against its full render in tests/test_gpu_batch.py)."""

import os
import socket
import tempfile
from datetime import timedelta

import numpy as np

from minirender_b200 import shard


def test_row_bands_cover_the_image():
    for height in (0, 1, 7, 1080):
        for world in (1, 2, 3, 8):
            bands = shard.row_bands(height, world)
            assert len(bands) == world and bands[0][0] == 0 and bands[-1][1] == height
            assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
            sizes = [e - b for b, e in bands]
            assert max(sizes) - min(sizes) <= 1


def test_partition_jobs_is_exact_and_balanced():
    rng = np.random.default_rng(4)
    costs = [int(c) for c in np.exp(rng.uniform(10, 20, 97))]
    for world in (1, 2, 4, 8):
        shares = shard.partition_jobs(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        # LPT bound: max load <= 4/3 of the optimum, and the optimum >= max(mean, largest job)
        lower = max(sum(costs) / world, max(costs))
        assert max(loads) <= 4 / 3 * lower + 1
    assert shard.partition_jobs(costs, 3) == shard.partition_jobs(costs, 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    from minirender_b200 import api, scene as sc
    from oracle import pyoracle
    try:
        doc = sc.cornell_box()
        o = pyoracle.OracleScene(doc.snapshot(), pyoracle.integrator("mis", 4, True, 3))
        render = api.RenderSettings(23, 17, 2, 5)

        def band(r, begin, end):
            img, _ = o.render(r.c(), threads=1, rows=(begin, end), statistics=False)
            return img

        frame = shard.render_frame_sharded(None, render, band_renderer=band)

        class Job:
            def __init__(self, k):
                self.render = api.RenderSettings(9 + 3 * k, 5 + k, 1 + k % 3, 11 + k)
                self.integrator = api.IntegratorSettings("mis", 2 + k % 4, True, 3)

        def alone(job):
            scene = pyoracle.OracleScene(doc.snapshot(), pyoracle.integrator(
                "mis", job.integrator.maximum_depth, True, 3))
            return scene.render(job.render.c(), threads=1, statistics=False)[0]

        jobs = [Job(k) for k in range(7)]
        rendered = []

        def batch(share):
            rendered.extend(share)
            return [alone(j) for j in share]

        images = shard.render_jobs_sharded(jobs, batch_renderer=batch)
        np.save(os.path.join(out, f"count{rank}.npy"), np.array([len(rendered)]))
        if rank == 0:
            ref, _ = o.render(render.c(), threads=1, statistics=False)
            np.save(os.path.join(out, "frame.npy"), frame)
            np.save(os.path.join(out, "frame_ref.npy"), ref)
            for k, (job, image) in enumerate(zip(jobs, images)):
                np.save(os.path.join(out, f"job{k}.npy"), image)
                np.save(os.path.join(out, f"job{k}_ref.npy"), alone(job))
        else:
            assert frame is None and images is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_frame_and_jobs(oracle):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                           start_method="spawn")
        frame = np.load(os.path.join(out, "frame.npy"))
        assert np.array_equal(frame, np.load(os.path.join(out, "frame_ref.npy")))
        for k in range(7):
            assert np.array_equal(np.load(os.path.join(out, f"job{k}.npy")),
                                  np.load(os.path.join(out, f"job{k}_ref.npy")))
        counts = [int(np.load(os.path.join(out, f"count{r}.npy"))[0]) for r in range(2)]
        assert sum(counts) == 7 and min(counts) >= 1


def test_partition_with_more_ranks_than_jobs():
    assert shard.partition_jobs([], 4) == [[], [], [], []]
    shares = shard.partition_jobs([5, 9, 1], 8)
    assert sorted(i for s in shares for i in s) == [0, 1, 2]
    assert sum(1 for s in shares if s) == 3 and all(len(s) <= 1 for s in shares)


def _worker_sparse(rank, world, port, out):
    # Three ranks, a two-row frame and two jobs: rank 2 holds an empty row band and no job.
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    from minirender_b200 import api, scene as sc
    from oracle import pyoracle
    try:
        doc = sc.cornell_box()
        o = pyoracle.OracleScene(doc.snapshot(), pyoracle.integrator("mis", 3, True, 3))
        render = api.RenderSettings(6, 2, 2, 9)
        seen = []

        def band(r, begin, end):
            seen.append((begin, end))
            img, _ = o.render(r.c(), threads=1, rows=(begin, end), statistics=False)
            return np.asarray(img)[: end - begin].reshape(end - begin, r.width, 3)

        frame = shard.render_frame_sharded(None, render, band_renderer=band)

        class Job:
            def __init__(self, k):
                self.render = api.RenderSettings(4 + k, 3, 1, 21 + k)
                self.integrator = api.IntegratorSettings("mis", 3, True, 3)

        def alone(job):
            return o.render(job.render.c(), threads=1, statistics=False)[0]

        jobs = [Job(0), Job(1)]
        rendered = []

        def batch(share):
            rendered.extend(share)
            return [alone(j) for j in share]

        images = shard.render_jobs_sharded(jobs, batch_renderer=batch)
        np.save(os.path.join(out, f"sparse{rank}.npy"), np.array([len(rendered), *seen[0]]))
        if rank == 0:
            np.save(os.path.join(out, "sparse_frame.npy"), frame)
            np.save(os.path.join(out, "sparse_frame_ref.npy"),
                    o.render(render.c(), threads=1, statistics=False)[0])
            for k, (job, image) in enumerate(zip(jobs, images)):
                np.save(os.path.join(out, f"sparse_job{k}.npy"), image)
                np.save(os.path.join(out, f"sparse_job{k}_ref.npy"), alone(job))
    finally:
        dist.destroy_process_group()


def test_three_gloo_ranks_with_an_empty_band_and_no_job(oracle):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_worker_sparse, args=(3, _free_port(), out), nprocs=3, join=True,
                           start_method="spawn")
        assert np.array_equal(np.load(os.path.join(out, "sparse_frame.npy")),
                              np.load(os.path.join(out, "sparse_frame_ref.npy")))
        for k in range(2):
            assert np.array_equal(np.load(os.path.join(out, f"sparse_job{k}.npy")),
                                  np.load(os.path.join(out, f"sparse_job{k}_ref.npy")))
        info = [np.load(os.path.join(out, f"sparse{r}.npy")) for r in range(3)]
        assert [int(i[0]) for i in info] == [1, 1, 0]  # jobs per rank (LPT: larger job first)
        assert [tuple(int(v) for v in i[1:]) for i in info] == [(0, 1), (1, 2), (2, 2)]
