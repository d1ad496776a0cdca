"""Writes the reference's own `studio` and `path-room` scenes as fixtures under tests/golden/scenes.

    python tests/golden/make_reference_scenes.py [REFERENCE_SCENE_DIRECTORY]

The directory defaults to the reference checkout's `scenes/` folder. Each scene is read with
``minirender_b200.scene_io.load_scene`` (the reference's scene JSON v1 + OBJ rules) and written
back with ``save_scene`` in this project's own serialisation (FP32 values printed with 9
significant digits, so they read back bit for bit). The fixtures let the tests pin the oracle to
outputs the reference itself recorded for these two scenes without needing the reference tree at
test time.
"""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from minirender_b200 import scene_io  # noqa: E402

SCENES = ("studio", "path-room", "studio-textured")


def main() -> None:
    source = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/scenes"
    out = os.path.join(HERE, "scenes")
    os.makedirs(out, exist_ok=True)
    for name in SCENES:
        doc = scene_io.load_scene(os.path.join(source, f"{name}.json"))
        path = os.path.join(out, f"{name}.json")
        scene_io.save_scene(doc, path)
        back = scene_io.load_scene(path)
        assert (back.snapshot().world_triangles() == doc.snapshot().world_triangles()).all()
        print(f"{path}: {doc.triangle_count} triangles")


if __name__ == "__main__":
    main()
