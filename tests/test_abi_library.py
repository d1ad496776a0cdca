"""The C-ABI library loads, exports every entry point the header declares, and fails loudly
(MR_CUDA_ERROR) instead of falling back to the CPU when no GPU is present. No GPU needed."""

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from minirender_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "minirender_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:mr_status|uint32_t|size_t)\s+(mr_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_abi.LIBRARY_PATH):
        from minirender_b200 import build
        build.build()
    return _abi.load_library()


def test_library_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIBRARY_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (mr_\w+)", out))
    assert set(names) <= exported, set(names) - exported
    assert set(names) == set(_abi.SIGNATURES), set(names) ^ set(_abi.SIGNATURES)


def test_struct_layouts_match_header_sizes():
    assert C.sizeof(_abi.MeshCorner) == 24
    assert C.sizeof(_abi.BvhNode) == 36
    assert C.sizeof(_abi.Ray) == 32
    assert C.sizeof(_abi.Hit) == 32


def test_abi_version(lib):
    assert lib.mr_abi_version() == 1


def test_display_image_is_host_side_reinhard(lib):
    from minirender_b200.api import display_image
    d = display_image(np.array([[[8, 2, 0.5]]], np.float32))
    assert d[0, 0, 0] == pytest.approx(8 / 9, abs=1e-7)
    with pytest.raises(_abi.MiniRenderError):
        display_image(np.array([[[np.inf, 0, 0]]], np.float32))


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="only meaningful without a GPU")
def test_no_cpu_fallback_without_gpu(lib):
    from minirender_b200.scene import cornell_box
    snap = cornell_box().snapshot()
    handle = C.c_void_p()
    status = lib.mr_scene_create(snap.desc_pointer(), None, C.byref(handle))
    assert status == 8  # MR_CUDA_ERROR
