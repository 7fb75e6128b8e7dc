"""Package two of the reference's example scenes for machines without the
reference checkout: misc/example_config/dense_sheet.json (the 6,273-vertex
sheet, model/dense_sheet.obj, of the README's "6K cloth" claim) and
misc/example_config/cloth_ball.json (the same sheet dropped on a ground
plane and a sphere).

For each scene the fixture holds the scene file's text and every mesh it
names as loaded by silk_physics_b200.headless.load_mesh (float32 vertices,
int32 triangles, before the scene's transform), so that
``scene_from_fixture`` can write the scene back out and the headless driver
(transforms, pin selection, configs) runs it exactly as it runs the
original files.

Run from the repository root (needs the reference checkout):
  python tests/golden/make_scene_assets.py
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from silk_physics_b200 import headless as H  # noqa: E402

REFERENCE = Path("/root/reference")
SCENES = ("dense_sheet", "cloth_ball")
OUT = HERE / "reference_scenes.npz"


def main():
    arrays = {}
    for name in SCENES:
        path = REFERENCE / "misc" / "example_config" / f"{name}.json"
        text = path.read_text()
        arrays[f"{name}/json"] = np.frombuffer(text.encode(), np.uint8)
        for o in json.loads(text)["objects"]:
            mesh = o["mesh"]
            key = f"mesh/{mesh}"
            if f"{key}/verts" in arrays:
                continue
            V, F = H.load_mesh(REFERENCE / mesh)
            arrays[f"{key}/verts"] = np.asarray(V, np.float32)
            arrays[f"{key}/faces"] = np.asarray(F, np.int32)
    np.savez_compressed(OUT, **arrays)
    print("written", OUT, sorted(arrays))


if __name__ == "__main__":
    main()
