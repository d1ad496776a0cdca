"""The GPU against outputs the reference itself recorded (the CPU side of these pins is
tests/test_reference_outputs.py, which checks the oracle against the same numbers):

  * the GPU binned-SAH builder on the reference's `studio` scene and its dense-floor variant:
    tree sizes of the binary tree it builds (the reference records 17 nodes, depth 4 and
    134,405 nodes, depth 20; docs/checkpoints/A2.1.md:44-47 of the MiniRender tree);
  * the path-room render, 160x160, 128 spp, depth 12, MIS, seed 101, on the GPU path: camera
    paths exact, scattering events within 0.05% and shadow rays within 0.3% of the reference's
    counts (docs/checkpoints/A2.3.md:43-46). The shadow-ray gap has one source, pinned by the
    second test: next-event estimation from points on the emitter quad itself (its material is
    diffuse with a black base colour, so its paths continue) toward light samples on the same
    quad. Sample and reference point are coplanar, so whether the light sample counts as on the
    reflection side is the sign of a dot product that is zero up to rounding: FP32 and FP64 decide
    it differently, the sample contributes nothing either way (black base colour), and only the
    count moves. On the rows whose camera rays do not see the emitter the GPU's first-vertex
    counts equal the oracle's exactly;
  * the MIS statistics table (tests/path_tests.cpp:291-341 of the reference): per-mode means over
    12 seeds x 2048 paths of the GPU's FP32 paths within 1e-5 relative of the reference's printed
    means, and variances within 1e-3 relative.
"""

import numpy as np
import pytest

from tests.test_reference_outputs import MIS_TABLE, PATH_ROOM, dense_floor, load, welford

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from minirender_b200 import api as a
    return a


@pytest.mark.parametrize("name,nodes,depth,triangles", [
    ("studio", 17, 4, 26), ("dense", 134_405, 20, 204_824)])
def test_gpu_builder_tree_sizes(api, oracle, name, nodes, depth, triangles):
    doc = load("studio") if name == "studio" else dense_floor(load("studio"))
    snap = doc.snapshot()
    built = api.Scene(snap)
    st = built.statistics()
    ref = oracle.OracleScene(snap)
    assert st["triangles"] == triangles
    print(f"{name}: GPU builder {st['nodes']} nodes, depth {st['maximum_depth']}; "
          f"reference builder {ref.bvh_counts()['nodes']} nodes; SAH {built.sah_cost():.4f} vs "
          f"{ref.sah_cost():.4f}")
    assert built.sah_cost() == pytest.approx(ref.sah_cost(), rel=0.02)
    assert st["nodes"] == pytest.approx(nodes, rel=0.01)
    assert abs(st["maximum_depth"] - depth) <= 1


def test_gpu_path_room_render_counters(api):
    snap = load("path-room").snapshot()
    tracer = api.PathTracer(api.Scene(snap), api.IntegratorSettings("mis", 12, True, 3))
    image, stats = tracer.render(api.RenderSettings(160, 160, 128, 101))
    assert np.isfinite(image).all() and image.mean() > 0
    assert stats["paths"] == PATH_ROOM["paths"]
    assert stats["scattering_events"] == pytest.approx(PATH_ROOM["scattering_events"], rel=5e-4)
    assert stats["shadow_rays"] == pytest.approx(PATH_ROOM["shadow_rays"], rel=3e-3)
    print({k: stats[k] for k in ("paths", "shadow_rays", "scattering_events")})


def test_gpu_path_room_first_vertex_counters_equal_oracle_away_from_the_emitter(api, oracle):
    snap = load("path-room").snapshot()
    g = api.Scene(snap)
    tracer = api.PathTracer(g, api.IntegratorSettings("mis", 1, False, 3))
    o = oracle.OracleScene(snap, oracle.integrator("mis", 1, False, 3))
    render = api.RenderSettings(160, 160, 8, 101)
    # Rows 0-19 see the emitter (instance 5); the rest do not.
    for rows in ((0, 20), (20, 160)):
        xs, ys = np.meshgrid(np.arange(160), np.arange(*rows))
        pixels = np.repeat(np.stack([xs.ravel(), ys.ravel()], 1), 8, axis=0).astype(np.uint32)
        samples = np.tile(np.arange(8, dtype=np.uint64), xs.size)
        _, _, rays = tracer.sample_pixels(render, pixels, samples, want_rays=True)
        hits, _ = g.intersect(rays[:, 0:3], rays[:, 3:6], rays[:, 6], rays[:, 7])
        on_emitter = int((hits["instance"] == 5).sum())
        _, gs = tracer.render_rows(render, rows[0], rows[1], statistics=True)
        _, cs = o.render(render.c(), rows=rows)
        print(f"rows {rows}: {on_emitter} camera hits on the emitter, shadow rays "
              f"{gs['shadow_rays']} vs {cs['shadow_rays']}")
        assert gs["scattering_events"] == cs["scattering_events"]
        if on_emitter == 0:
            assert gs["shadow_rays"] == cs["shadow_rays"]
        else:
            assert abs(gs["shadow_rays"] - cs["shadow_rays"]) <= on_emitter


@pytest.mark.parametrize("glossy", [False, True])
def test_gpu_mis_statistics_table(api, glossy):
    from tests.test_oracle_golden import direct_doc
    snap = direct_doc(glossy).snapshot()
    scene = api.Scene(snap)
    for mode, (mean_ref, var_ref) in MIS_TABLE[glossy].items():
        tracer = api.PathTracer(scene, api.IntegratorSettings(mode, 1, False, 3))
        seed_means = []
        for seed in range(17, 17 + 12):
            keys = np.zeros((2048, 3), np.uint64)
            keys[:, 0] = seed
            keys[:, 2] = np.arange(2048)
            rad, _ = tracer.trace([[0, 1, 0]] * 2048, [[0, -1, 0]] * 2048, 0, 10000, keys)
            seed_means.append(welford(rad[:, 0].astype(np.float64).tolist())[0])
        mean, variance = welford(seed_means)
        print(f"glossy={glossy} {mode}: mean {mean:.7g} (reference {mean_ref}), "
              f"variance {variance:.6g} (reference {var_ref})")
        assert mean == pytest.approx(mean_ref, rel=1e-5)
        assert variance == pytest.approx(var_ref, rel=1e-3)
