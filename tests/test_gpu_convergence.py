"""Converged images: a 16,384-spp GPU render agrees with the FP64 oracle's independent render
within Monte Carlo noise.

The GPU reference is 16 renders of 1,024 spp with seeds 1..16 (so every pixel has a standard
error from the spread of the 16 means); the oracle renders a band of rows at 2,048 spp as 16
renders of 128 spp with seeds 101..116. Different seeds make the two estimates independent. Bar:
per pixel and channel |gpu - oracle| <= 3 sqrt(se_gpu^2 + se_oracle^2) for at least 97% of the
band's values (with standard errors estimated from 16 batches about 1% exceed 3 sigma by
chance), and the band means within 3 combined standard errors."""

import os

import numpy as np
import pytest

from minirender_b200 import scene as sc

pytestmark = pytest.mark.gpu


def batch_moments(images):
    stack = np.stack([np.asarray(i, np.float64) for i in images])
    return stack.mean(0), stack.std(0, ddof=1) / np.sqrt(len(images))


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_16k_spp_gpu_reference_agrees_with_oracle(oracle, name):
    from minirender_b200 import api
    if name == "cornell":
        doc = sc.cornell_box()
    else:
        doc = sc.sphere_field(12, 6.0, 3, subdivisions=2)
        doc.camera = sc.Camera(position=(0.0, 3.0, 9.0), target=(0.0, 2.5, 0.0),
                               aperture_radius=0.05, focus_distance=8.0, vertical_fov_degrees=45.0)
    snap = doc.snapshot()
    width, height, rows = 32, 24, (10, 14)
    tracer = api.PathTracer(api.Scene(snap), api.IntegratorSettings("mis", 8, True, 3))
    gpu = [tracer.render(api.RenderSettings(width, height, 1024, seed), statistics=False)[0]
           for seed in range(1, 17)]
    g_mean, g_err = batch_moments(gpu)
    o = oracle.OracleScene(snap, oracle.integrator("mis", 8, True, 3))
    threads = max(1, (os.cpu_count() or 2) - 1)
    cpu = [o.render(api.RenderSettings(width, height, 128, seed).c(), threads=threads, rows=rows,
                    statistics=False)[0] for seed in range(101, 117)]
    c_mean, c_err = batch_moments(cpu)
    band_gpu, band_err = g_mean[rows[0]:rows[1]], g_err[rows[0]:rows[1]]
    sigma = np.sqrt(band_err ** 2 + c_err ** 2)
    within = np.abs(band_gpu - c_mean) <= 3 * sigma + 1e-7
    assert within.mean() >= 0.97, within.mean()
    mean_sigma = np.sqrt((band_err ** 2).sum() + (c_err ** 2).sum()) / band_gpu.size
    assert abs(band_gpu.mean() - c_mean.mean()) <= 3 * mean_sigma
