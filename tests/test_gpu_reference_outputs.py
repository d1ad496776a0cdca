"""The GPU against outputs the reference itself recorded (the CPU side of these pins is
tests/test_reference_outputs.py, which checks the oracle against the same numbers):

  * the GPU binned-SAH builder on the reference's `studio` scene and its dense-floor variant:
    tree sizes of the binary tree it builds (the reference records 17 nodes, depth 4 and
    134,405 nodes, depth 20; docs/checkpoints/A2.1.md:44-47 of the MiniRender tree);
  * the path-room render, 160x160, 128 spp, depth 12, MIS, seed 101, on the GPU path: camera
    paths exact, shadow rays and scattering events within 0.1% of the reference's counts
    (docs/checkpoints/A2.3.md:43-46). The CPU oracle is within 0.05% of them; FP32 moves a few
    more decisions that sit within rounding of their thresholds;
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
    for key in ("shadow_rays", "scattering_events"):
        assert stats[key] == pytest.approx(PATH_ROOM[key], rel=1e-3), (key, stats[key])
    print({k: stats[k] for k in ("paths", "shadow_rays", "scattering_events")})


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
