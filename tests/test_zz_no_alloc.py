"""The allocation-free entry point mr_trace_paths_static, called through the C ABI.

Some callers cannot allocate device memory while rendering (a server that has reserved its
whole HBM budget in its own pool, or a loop that must not pay the device synchronisation an
allocation can cause). mr_trace_paths_static serves them from one fixed array inside the
library. This file checks, on two calls in a row, that it returns exactly what the allocating
entry point mr_trace_paths returns for the same rays and sampler keys (both run the same
kernels on the same per-path state, so the tolerance is zero), that the second call is not
disturbed by what the first one left in the shared array, that after the zero-length warm-up a
call leaves the device's free memory unchanged, that a ray just outside the unit-length tolerance
is rejected by both entry points alike, and that the batch limit is enforced.
The test buffers themselves come from torch; only the entry point under test allocates nothing.
It is collected last so a failing run that stops at the first failure has run everything else.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _paths(count, seed):
    rng = np.random.default_rng(seed)
    origins = np.zeros((count, 3), np.float32) + np.float32([0.0, 0.5, 1.87])
    targets = rng.uniform([-0.45, 0.05, -0.45], [0.45, 0.95, 0.45], (count, 3)).astype(np.float32)
    d = targets - origins
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    keys = np.zeros((count, 3), np.uint64)
    keys[:, 0] = seed
    keys[:, 1] = np.arange(count) % 997
    keys[:, 2] = np.arange(count)
    return origins, d, keys


def _static_call(lib, scene, settings, rays, keys, count, check_memory=False):
    import torch
    d_rays = torch.from_numpy(rays.reshape(-1).copy()).cuda()
    d_keys = torch.from_numpy(keys.reshape(-1).view(np.int64).copy()).cuda()
    d_out = torch.full((count * 3,), -7.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    status = lib.mr_trace_paths_static(scene.handle, C.byref(settings), C.c_void_p(d_rays.data_ptr()),
                                       C.c_void_p(d_keys.data_ptr()), count,
                                       C.c_void_p(d_out.data_ptr()), None)
    if check_memory:
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, "the call changed free device memory"
    return status, d_out.cpu().numpy().reshape(count, 3)


def _warm_up(lib, scene, settings):
    """The documented warm-up: a zero-length call resolves (and places) the static array."""
    assert lib.mr_trace_paths_static(scene.handle, C.byref(settings), None, None, 0, None, None) == 0


def test_static_entry_matches_allocating_entry_twice():
    from minirender_b200 import _abi, api
    from minirender_b200.api import pack_rays
    from minirender_b200.scene import cornell_box

    lib = _abi.load_library()
    scene = api.Scene(cornell_box().snapshot())
    integrator = api.IntegratorSettings("mis", 8, True, 3)
    tracer = api.PathTracer(scene, integrator)
    settings = integrator.c()
    _warm_up(lib, scene, settings)
    for count, seed in ((12000, 31), (5000, 32)):  # the second call is smaller than the first
        origins, dirs, keys = _paths(count, seed)
        expected, _ = tracer.trace(origins, dirs, 0.0, np.inf, keys)
        rays = pack_rays(origins, dirs, 0.0, np.inf)
        status, got = _static_call(lib, scene, settings, rays, keys, count, check_memory=True)
        assert status == 0, _abi.STATUS_NAMES.get(status)
        assert got.shape == expected.shape
        assert np.array_equal(got, expected)
        assert np.all(got >= 0) and got.mean() > 0


def test_static_entry_rejects_batches_over_the_limit():
    from minirender_b200 import _abi, api
    from minirender_b200.api import pack_rays
    from minirender_b200.scene import cornell_box

    lib = _abi.load_library()
    scene = api.Scene(cornell_box().snapshot())
    settings = api.IntegratorSettings().c()
    count = 16385
    origins, dirs, keys = _paths(count, 5)
    status, _ = _static_call(lib, scene, settings, pack_rays(origins, dirs, 0.0, np.inf), keys, count)
    assert status == 1  # MR_INVALID_ARGUMENT
    buf = C.create_string_buffer(256)
    lib.mr_last_error(buf, 256)
    assert b"MR_STATIC_MAX_PATHS" in buf.value


def test_static_entry_rejects_the_rays_the_allocating_entry_rejects():
    from minirender_b200 import _abi, api
    from minirender_b200.api import pack_rays
    from minirender_b200.scene import cornell_box

    lib = _abi.load_library()
    scene = api.Scene(cornell_box().snapshot())
    integrator = api.IntegratorSettings("mis", 4, True, 3)
    tracer = api.PathTracer(scene, integrator)
    settings = integrator.c()
    _warm_up(lib, scene, settings)
    origins, dirs, keys = _paths(64, 7)
    # Squared lengths 1 +- 0.99e-4 pass and 1 +- 1.01e-4 fail, with the check in FP64.
    for scale, accepted in ((1.0 + 0.495e-4, True), (1.0 - 0.495e-4, True),
                            (1.0 + 0.505e-4, False), (1.0 - 0.505e-4, False)):
        d = dirs.copy()
        d[5] = (d[5].astype(np.float64) * scale).astype(np.float32)
        d2 = float(np.sum(d[5].astype(np.float64) ** 2))
        assert (abs(d2 - 1) <= 1e-4) == accepted
        try:
            tracer.trace(origins, d, 0.0, np.inf, keys)
            host_ok = True
        except api.MiniRenderError:
            host_ok = False
        status, _ = _static_call(lib, scene, settings, pack_rays(origins, d, 0.0, np.inf), keys, 64)
        assert host_ok == accepted and (status == 0) == accepted, (scale, host_ok, status)
