"""Headless JSON scene driver: mesh loaders, transforms, pin selection, scene
parsing (CPU), and a generated scene run against the same objects stepped
directly through the API (GPU)."""
import json
import math
import struct

import numpy as np
import pytest

from silk_physics_b200 import headless as H
from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

QUAD_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
QUAD_F = np.array([[0, 1, 2], [0, 2, 3]], np.int32)


def _tri_set(V, F):
    return {tuple(sorted(tuple(np.round(V[i], 6)) for i in f)) for f in F}


def _write_all(tmp_path):
    p = {}
    obj = tmp_path / "q.obj"
    obj.write_text("# quad\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1/1 2/2 3/3 4/4\n")
    p["obj"] = obj
    off = tmp_path / "q.off"
    off.write_text("OFF\n4 1 0\n0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    p["off"] = off
    ply = tmp_path / "q_ascii.ply"
    ply.write_text("ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\n"
                   "property float z\nelement face 1\nproperty list uchar int vertex_indices\n"
                   "end_header\n0 0 0\n1 0 0\n1 1 0\n0 1 0\n4 0 1 2 3\n")
    p["ply_ascii"] = ply
    plyb = tmp_path / "q_bin.ply"
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\n"
            "property float y\nproperty float z\nelement face 2\n"
            "property list uchar int vertex_indices\nend_header\n").encode()
    body = b"".join(struct.pack("<3f", *v) for v in QUAD_V)
    body += b"".join(struct.pack("<B3i", 3, *f) for f in QUAD_F)
    plyb.write_bytes(head + body)
    p["ply_bin"] = plyb
    stl = tmp_path / "q.stl"
    rec = b"".join(struct.pack("<3f", 0, 0, 1) + b"".join(struct.pack("<3f", *QUAD_V[i]) for i in f)
                   + struct.pack("<H", 0) for f in QUAD_F)
    stl.write_bytes(b"\0" * 80 + struct.pack("<I", 2) + rec)
    p["stl"] = stl
    stla = tmp_path / "qa.stl"
    lines = ["solid q"]
    for f in QUAD_F:
        lines += ["facet normal 0 0 1", "outer loop"]
        lines += [f"vertex {QUAD_V[i][0]} {QUAD_V[i][1]} {QUAD_V[i][2]}" for i in f]
        lines += ["endloop", "endfacet"]
    lines.append("endsolid q")
    stla.write_text("\n".join(lines) + "\n")
    p["stl_ascii"] = stla
    return p


def test_mesh_loaders_agree(tmp_path):
    ref = _tri_set(QUAD_V, QUAD_F)
    for name, path in _write_all(tmp_path).items():
        V, F = H.load_mesh(path)
        assert _tri_set(V, F) == ref, name


def test_transform_composition():
    V = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], np.float32)
    # Rz(pi/2) after scaling by 2, then translation.
    out = H.apply_transform(V, {"translation": [0, 0, 1], "rotation_euler_deg": [0, 0, math.pi / 2],
                                "scale": 2.0})
    np.testing.assert_allclose(out, [[0, 2, 1], [-2, 0, 1]], atol=1e-6)
    # Rz Ry Rx order: x-rotation applied first.
    R = H.rotation(0.3, -0.2, 0.7)
    cx, sx = math.cos(0.3), math.sin(0.3)
    cy, sy = math.cos(-0.2), math.sin(-0.2)
    cz, sz = math.cos(0.7), math.sin(0.7)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    np.testing.assert_allclose(R, Rz @ Ry @ Rx)
    # Per-axis scale.
    out = H.apply_transform(V, {"scale": [1, 3, 1]})
    np.testing.assert_allclose(out, [[1, 0, 0], [0, 3, 0]])


def test_pin_selection_bbox():
    V, _ = S.grid_sheet(5, side=1.0, z=0.0)
    pins = H.select_pins(V, {"min": [0.6, 0.6, -1], "max": [-1, 0.4, 1]})  # swapped on x
    assert set(pins.tolist()) == {i for i, v in enumerate(V) if v[1] >= 0.4 and v[0] <= 0.6}


def test_malformed_meshes_raise_clear_errors(tmp_path):
    """Truncated or inconsistent mesh files fail with the file, the format
    and the reason, not with an index or buffer error from the parser."""
    cases = {
        "short.obj": ("v 0 0\nf 1 2 3\n", "vertex needs three coordinates"),
        "oob.obj": ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n", "face index out of range"),
        "noy.ply": ("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\n"
                    "end_header\n0\n", "without properties y, z"),
        "bad.off": ("OFF\n3 1 0\n0 0 0\n1 0 0\n", "malformed OFF file"),
    }
    for name, (text, msg) in cases.items():
        f = tmp_path / name
        f.write_text(text)
        with pytest.raises(ValueError, match=msg):
            H.load_mesh(f)
    stl = tmp_path / "short.stl"
    stl.write_bytes(b"\0" * 80 + struct.pack("<I", 5))
    with pytest.raises(ValueError, match="declares 5 triangles but holds 0"):
        H.load_mesh(stl)
    with pytest.raises(ValueError, match="unsupported mesh format"):
        H.load_mesh(tmp_path / "x.xyz")


def test_scene_with_missing_mesh_names_it(tmp_path):
    scene = tmp_path / "scene.json"
    scene.write_text(json.dumps({"global": {}, "objects": [
        {"type": "cloth", "name": "a", "mesh": "nope.obj"}]}))
    with pytest.raises(FileNotFoundError, match="'nope.obj' not found"):
        H.load_scene(scene)


def _scene_files(tmp_path, steps=3):
    V, F = S.grid_sheet(16, side=0.5, z=0.0, jitter=1e-4, seed=3)
    with open(tmp_path / "sheet.obj", "w") as f:
        for v in V:
            f.write(f"v {v[0]:.9g} {v[1]:.9g} {v[2]:.9g}\n")
        for t in F:
            f.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
    SV, SF = S.icosphere(2, radius=0.2)
    with open(tmp_path / "ball.off", "w") as f:
        f.write(f"OFF\n{len(SV)} {len(SF)} 0\n")
        for v in SV:
            f.write(f"{v[0]:.9g} {v[1]:.9g} {v[2]:.9g}\n")
        for t in SF:
            f.write(f"3 {t[0]} {t[1]} {t[2]}\n")
    cfg = {
        "global": {"dt": 1.0 / 60.0, "max_outer_iteration": 50, "max_inner_iteration": 30,
                   "acceleration": [0.0, 0.0, -9.8], "total_steps": steps},
        "objects": [
            {"type": "cloth", "name": "sheet", "mesh": "sheet.obj",
             "cloth": {"elastic_stiffness": 120.0, "bending_stiffness": 1e-4, "density": 0.1,
                       "damping": 0.01},
             "collision": {"enabled": True, "self_collision": True, "group": 1,
                           "restitution": 0.3, "friction": 0.3},
             "transform": {"translation": [0, 0, 0.23], "rotation_euler_deg": [0.1, 0, 0],
                           "scale": 1.0},
             "pin_selection": {"bbox": {"min": [-1, 0.2, -1], "max": [-0.2, 1, 1]}}},
            {"type": "obstacle", "name": "ball", "mesh": "ball.off",
             "collision": {"enabled": True, "self_collision": False, "group": 1},
             "transform": {"translation": [0, 0, 0], "rotation_euler_deg": [0, 0, 0],
                           "scale": [1.0, 1.0, 1.0]},
             "angular_velocity_deg_s": [0.0, 0.0, 90.0]},
        ],
    }
    path = tmp_path / "scene.json"
    path.write_text(json.dumps(cfg))
    return path, cfg


def test_scene_parsing(tmp_path):
    path, cfg = _scene_files(tmp_path)
    g, objs = H.load_scene(path)
    assert g["total_steps"] == 3
    sheet, ball = objs
    assert sheet.kind == "cloth" and ball.kind == "obstacle"
    assert len(sheet.pins) > 0
    assert abs(sheet.cfg.elastic_stiffness - 120.0) < 1e-6 and sheet.coll.group == 1
    np.testing.assert_allclose(ball.omega, [0, 0, math.pi / 2])
    assert np.all(H.select_pins(sheet.verts, cfg["objects"][0]["pin_selection"]["bbox"])
                  == sheet.pins)


@pytest.mark.gpu
def test_headless_run_equals_direct_api(tmp_path):
    path, _ = _scene_files(tmp_path, steps=4)
    out = tmp_path / "out.npz"
    objs, wall = H.run(path, str(out), log=None)
    res = np.load(out)
    assert res["sheet/positions"].shape == (5, 256, 3)
    assert res["ball/positions"].shape[0] == 5  # rotating obstacle recorded
    # The same objects stepped directly.
    g, objs2 = H.load_scene(path)
    w = N.World()
    assert w.init() and w.set_global_config(H.global_config(g))
    sheet, ball = objs2
    r, hc = w.add_cloth(sheet.cfg, sheet.coll, sheet.verts, sheet.faces, sheet.pins)
    r2, hb = w.add_obstacle(ball.coll, ball.verts, ball.faces)
    assert r and r2
    V = ball.verts.copy()
    x = np.zeros(sheet.verts.size, np.float32)
    for k in range(4):
        R = H.rotation(*(g["dt"] * ball.omega))
        V = ((V.astype(np.float64) - ball.pivot) @ R.T + ball.pivot).astype(np.float32)
        assert w.set_obstacle_position(hb, V.ravel())
        assert w.solver_step()
        assert w.get_cloth_position(hc, x)
        np.testing.assert_array_equal(res["sheet/positions"][k + 1], x.reshape(-1, 3))
        np.testing.assert_array_equal(res["ball/positions"][k + 1], V)
    # Pinned vertices stayed put.
    np.testing.assert_array_equal(res["sheet/positions"][-1][sheet.pins], sheet.verts[sheet.pins])


REFERENCE = __import__("pathlib").Path("/root/reference")
EXAMPLES = REFERENCE / "misc" / "example_config"
FIXTURE = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "reference_scenes.npz"


def reference_scene(name, directory):
    """Write one packaged reference scene (tests/golden/reference_scenes.npz)
    into `directory`; returns the scene file path."""
    d = dict(np.load(FIXTURE))
    text = bytes(d[f"{name}/json"]).decode()
    meshes = {o["mesh"]: (d[f"mesh/{o['mesh']}/verts"], d[f"mesh/{o['mesh']}/faces"])
              for o in json.loads(text)["objects"]}
    return H.write_scene(directory, name, text, meshes)


@pytest.mark.skipif(not EXAMPLES.exists(), reason="reference checkout absent")
def test_every_reference_example_scene_loads(monkeypatch):
    """All seven scene files of misc/example_config parse with the reference's
    meshes (paths relative to the reference root, as its demo resolves them):
    objects and configs read, transforms applied, pins selected where a pin
    box is given, and every cloth mesh passes the host mesh checks and
    partitions into MAS banks."""
    monkeypatch.chdir(REFERENCE)
    files = sorted(EXAMPLES.glob("*.json"))
    assert [p.stem for p in files] == ["bunny_and_cloth", "cloth_ball", "cloth_on_the_ground",
                                       "default", "default_gpu", "dense_sheet", "simple_sheet"]
    for p in files:
        g, objs = H.load_scene(p)
        cfg = json.loads(p.read_text())
        gc = H.global_config(g)
        assert gc.dt == pytest.approx(cfg["global"]["dt"])
        assert gc.max_inner_iteration == cfg["global"]["max_inner_iteration"]
        assert len(objs) == len(cfg["objects"])
        for o, spec in zip(objs, cfg["objects"]):
            assert o.kind == spec["type"] and len(o.verts) > 0 and len(o.faces) > 0
            assert np.isfinite(o.verts).all()
            if (spec.get("pin_selection") or {}).get("bbox"):
                assert len(o.pins) > 0, (p.name, o.name)
            if o.kind == "cloth":
                perm, offs = N.partition_mesh(o.verts, o.faces)
                assert sorted(perm.tolist()) == list(range(len(o.verts)))
                assert offs[-1] == len(o.verts)


def test_packaged_reference_scenes(tmp_path, monkeypatch):
    """The packaged dense_sheet and cloth_ball scenes rebuild the reference's
    objects exactly (compared with the original files where the checkout is
    present)."""
    for name, nobj in (("dense_sheet", 1), ("cloth_ball", 3)):
        g, objs = H.load_scene(reference_scene(name, tmp_path / name))
        assert len(objs) == nobj and objs[0].kind == "cloth" and len(objs[0].verts) == 6273
        if name == "dense_sheet":
            assert len(objs[0].pins) == 162
        if EXAMPLES.exists():
            monkeypatch.chdir(REFERENCE)
            g2, ref = H.load_scene(EXAMPLES / f"{name}.json")
            assert g == g2
            for a, b in zip(objs, ref):
                np.testing.assert_array_equal(a.verts, b.verts)
                np.testing.assert_array_equal(a.faces, b.faces)
                np.testing.assert_array_equal(a.pins, b.pins)
