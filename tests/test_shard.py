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
