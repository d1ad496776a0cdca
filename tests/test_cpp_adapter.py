"""The header-only C++ adapter (include/minirender_b200.hpp) compiles and links against the
library the way a MiniRender caller would use it; without a GPU its calls throw instead of
falling back to the CPU."""

import os
import subprocess
import tempfile

import pytest

from minirender_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include "minirender_b200.hpp"
#include <algorithm>
#include <cstdio>
#include <stdexcept>

int main() {
    // One triangle, pinhole camera: the smallest snapshot.
    const float positions[] = {0, 0, 0, 1, 0, 0, 0, 1, 0};
    mr_mesh_corner corners[3] = {{0, {0, 0, 1}, {0, 0}}, {1, {0, 0, 1}, {1, 0}}, {2, {0, 0, 1}, {0, 1}}};
    mr_mesh mesh{positions, 3, corners, 1};
    mr_material material{MR_MATERIAL_DIFFUSE, {0.7f, 0.7f, 0.7f}, {0, 0, 0}, 0.35f, 1.5f, 1};
    mr_instance instance{0, 0, {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}, {1, 0, 0, 0, 1, 0, 0, 0, 1}};
    mr_scene_desc desc{};
    desc.camera = {{0, 0, 3}, {0, 0, 0}, {0, 1, 0}, 45, 0.05f, 100, 0, 4};
    desc.environment[0] = desc.environment[1] = desc.environment[2] = 1;
    desc.meshes = &mesh; desc.mesh_count = 1;
    desc.materials = &material; desc.material_count = 1;
    desc.instances = &instance; desc.instance_count = 1;
    try {
        auto scene = std::make_shared<const minirender_b200::Scene>(desc);
        minirender_b200::PathTracer tracer(scene);
        auto image = tracer.render({8, 8, 4, 1});
        std::printf("rendered %zu x %zu mean %f\n", image.width, image.height, image.rgb[0]);
        auto band = tracer.render_rows({8, 8, 4, 1}, 2, 5);
        auto batch = minirender_b200::render_batch({{scene, {8, 8, 4, 1}}, {scene, {5, 3, 2, 9}}});
        minirender_b200::RenderServer server;
        const uint64_t job = server.submit(scene, {8, 8, 4, 1});
        if (!server.wait_for(job, std::chrono::milliseconds(60000))) return 4;
        auto served = server.result(job);
        server.release(job);
        const bool same = band.rgb.size() == 3 * 8 * 3 &&
                          std::equal(band.rgb.begin(), band.rgb.end(), image.rgb.begin() + 3 * 8 * 2) &&
                          batch[0].rgb == image.rgb && served.rgb == image.rgb;
        std::printf("batch and served images %s\n", same ? "match" : "differ");
        return same ? 0 : 5;
    } catch (const std::runtime_error& e) {
        std::printf("runtime_error: %s\n", e.what());
        return 3;
    }
}
"""


def test_cpp_adapter_compiles_links_and_reports_errors():
    if not os.path.exists(_abi.LIBRARY_PATH):
        from minirender_b200 import build
        build.build()
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "caller.cpp")
        exe = os.path.join(tmp, "caller")
        with open(src, "w") as f:
            f.write(PROGRAM)
        lib_dir = os.path.dirname(_abi.LIBRARY_PATH)
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), src,
                        "-o", exe, f"-L{lib_dir}", "-lminirender_b200",
                        f"-Wl,-rpath,{lib_dir}"], check=True)
        result = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        if os.path.exists("/dev/nvidia0"):
            assert result.returncode == 0, result.stdout + result.stderr
            assert "rendered 8 x 8" in result.stdout and "match" in result.stdout
        else:
            assert result.returncode == 3 and "CUDA" in result.stdout, result.stdout
