"""The render command on the GPU: ``python -m minirender_b200.render_cli scene.json out-prefix``.

Same arguments, outputs and report as the reference's ``minirender_cli --render``
(src/app/render_cli.cpp:46-181): a scene JSON v1 file, an output prefix (a trailing .png or .exr
is dropped), options ``--width --height --spp --depth --mode mis|bsdf|light --seed --exposure
--no-rr --rr-depth --threads --tile --batch``; the render runs as a RenderSession with progress
lines on stderr, then ``prefix.exr`` (linear) and ``prefix.png`` (display_image with the exposure,
sRGB) are written and the statistics printed. ``--integrator sppm`` and its options are rejected:
SPPM is not part of this path tracer. ``--trace-normals scene.json out.png`` is the geometry
diagnostic of src/app/cli.cpp:60-97.
"""

from __future__ import annotations

import os
import sys
import time

from . import api
from .image_io import write_exr, write_png
from .scene_io import load_scene

USAGE = ("Usage: --render scene.json output-prefix [--width N --height N --spp N --depth N "
         "--mode mis|bsdf|light --seed N --exposure EV --no-rr --rr-depth N --threads N --tile N "
         "--batch N]")


def _number(text: str, kind):
    try:
        value = kind(text)
    except ValueError:
        raise ValueError(f"Invalid number: {text}") from None
    if kind is int and value < 0:
        raise ValueError(f"Invalid number: {text}")
    return value


def run(argv: list[str]) -> int:
    if len(argv) < 2:
        raise ValueError(USAGE)
    render = api.RenderSettings()
    integrator = api.IntegratorSettings()
    session = api.SessionSettings()
    exposure = 0.0
    options = argv[2:]
    i = 0
    while i < len(options):
        option = options[i]
        if option == "--no-rr":
            integrator.russian_roulette = False
            i += 1
            continue
        if i + 1 >= len(options):
            raise ValueError(f"Render option is missing its value: {option}")
        value = options[i + 1]
        i += 2
        if option == "--width":
            render.width = _number(value, int)
        elif option == "--height":
            render.height = _number(value, int)
        elif option == "--spp":
            render.samples_per_pixel = _number(value, int)
        elif option == "--depth":
            integrator.maximum_depth = _number(value, int)
        elif option == "--rr-depth":
            integrator.roulette_depth = _number(value, int)
        elif option == "--threads":
            session.threads = _number(value, int)
        elif option == "--tile":
            session.tile_size = _number(value, int)
        elif option == "--batch":
            session.batch_samples = _number(value, int)
        elif option == "--seed":
            render.seed = _number(value, int)
        elif option == "--mode":
            if value not in ("mis", "bsdf", "light"):
                raise ValueError("Sampling mode must be bsdf, light or mis")
            integrator.mode = value
        elif option == "--exposure":
            exposure = _number(value, float)
        elif option in ("--integrator", "--photons", "--radius", "--alpha", "--sppm-memory-mb"):
            if option == "--integrator" and value == "path":
                continue
            raise ValueError("SPPM is not supported by this path tracer")
        else:
            raise ValueError(f"Unknown render option: {option}")
    if not (abs(exposure) <= 64):
        raise ValueError("Exposure must be finite and in [-64,64]")
    scene = api.Scene(load_scene(argv[0]).snapshot())
    start = time.perf_counter()
    job = api.RenderSession()
    job.start(scene, render, integrator, session)
    while not job.wait_for(200):
        p = job.progress()
        print(f"progress: {p['state']} {p['recorded_samples']}/{p['total_samples']}", file=sys.stderr)
    job.wait()
    progress = job.progress()
    if progress["state"] != "completed":
        raise RuntimeError(progress["error"] or "Render did not complete")
    image = job.result()
    finished = time.perf_counter()
    prefix = argv[1]
    if prefix.endswith((".png", ".exr")):
        prefix = prefix[:-4]
    parent = os.path.dirname(prefix)
    if parent:
        os.makedirs(parent, exist_ok=True)
    write_exr(prefix + ".exr", image)
    write_png(prefix + ".png", api.display_image(image, exposure))
    s = progress["statistics"]
    print(f"GPU path render complete\nmode: {integrator.mode}\n"
          f"resolution: {render.width}x{render.height}\nspp: {render.samples_per_pixel}\n"
          f"paths: {s['paths']}\nrecorded samples: {progress['recorded_samples']}\n"
          f"shadow rays: {s['shadow_rays']}\nscattering events: {s['scattering_events']}\n"
          f"medium scattering events: {s['medium_scattering_events']}\n"
          f"triangle tests: {s['triangle_tests']}\n"
          f"elapsed ms: {1e3 * (finished - start):.1f}\nEXR and PNG saved.")
    job.close()
    return 0


def trace_normals(scene_path: str, output: str) -> int:
    """The --trace-normals geometry diagnostic (src/app/cli.cpp:60-97): one primary ray through
    each pixel centre of a 256x256 image (pinhole, aspect 1, clip interval near/cos..far/cos),
    the world-space shading normal of the nearest hit mapped to n * 0.5 + 0.5 (black on a miss),
    written as PNG, with the BVH statistics, build and trace times and the query counters."""
    import numpy as np
    doc = load_scene(scene_path)
    snap = doc.snapshot()
    start = time.perf_counter()
    scene = api.Scene(snap)
    built = time.perf_counter()
    size = 256
    c = doc.camera
    f32 = np.float32
    position = np.asarray(c.position, f32)
    forward = np.asarray(c.target, f32) - position
    forward = (forward / np.linalg.norm(forward)).astype(f32)
    right = np.cross(forward, np.asarray(c.up, f32))
    right = (right / np.linalg.norm(right)).astype(f32)
    up = np.cross(right, forward).astype(f32)
    half = f32(np.tan(np.radians(c.vertical_fov_degrees) * 0.5))
    centres = (np.arange(size, dtype=f32) + f32(0.5)) / f32(size)
    v, u = np.meshgrid(centres, centres, indexing="ij")
    d = (forward + ((f32(2) * u - f32(1)) * half)[..., None] * right +
         ((f32(1) - f32(2) * v) * half)[..., None] * up).reshape(-1, 3)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(f32)
    cosine = d @ forward
    hits, counters = scene.intersect(np.broadcast_to(position, d.shape), d,
                                     c.near_plane / cosine, c.far_plane / cosine)
    # SceneBvh::surface_hit's shading normal (src/render/bvh.cpp:302-330): barycentric sum of
    # the unit world corner normals, oriented to the geometric normal's side.
    visible = [o for o in doc.objects if o.visible]
    image = np.zeros((size * size, 3), f32)
    world = snap.world_triangles().astype(np.float64)
    hit = np.nonzero(hits["primitive"] != 0xFFFFFFFF)[0]
    for i in hit:
        obj = visible[int(hits["instance"][i])]
        mesh = doc.meshes[obj.mesh]
        n_to_w = obj.transform.normal_matrix().astype(np.float64).T  # column-major storage
        corners = mesh.corner_normals[int(hits["triangle"][i])].astype(np.float64)
        tri = world[int(hits["primitive"][i])]
        geometric = np.cross(tri[1] - tri[0], tri[2] - tri[0])
        geometric /= np.linalg.norm(geometric)
        if np.linalg.det(obj.transform.matrix()[:3, :3].astype(np.float64)) < 0:
            geometric = -geometric
        shading = np.zeros(3)
        for k in range(3):
            w = n_to_w @ corners[k]
            shading += float(hits["barycentric"][i][k]) * w / np.linalg.norm(w)
        if shading @ shading < 1e-24:
            shading = geometric
        else:
            shading /= np.linalg.norm(shading)
            if shading @ geometric < 0:
                shading = -shading
        image[i] = shading * 0.5 + 0.5
    finished = time.perf_counter()
    write_png(output, image.reshape(size, size, 3))
    stats = scene.statistics()
    print(f"geometry diagnostic: world-space shading normals\ntriangles: {stats['triangles']}\n"
          f"nodes: {stats['nodes']}\nleaves: {stats['leaves']}\n"
          f"maximum depth: {stats['maximum_depth']}\nbuild ms: {1e3 * (built - start):.3f}\n"
          f"trace ms: {1e3 * (finished - built):.3f}\n"
          f"bounds tests: {counters['bounds_tests']}\ntriangle tests: {counters['triangle_tests']}")
    return 0


def main() -> int:
    args = sys.argv[1:]
    try:
        if args and args[0] == "--trace-normals":
            if len(args) != 3:
                raise ValueError("Usage: --trace-normals scene.json output.png")
            return trace_normals(args[1], args[2])
        if args and args[0] == "--render":
            args = args[1:]
        return run(args)
    except (ValueError, RuntimeError, api.MiniRenderError) as error:
        print(f"error: {error}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
