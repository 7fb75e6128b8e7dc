"""Headless scene driver: run a JSON scene in the reference's config format
(demo/src/json_parse.cpp, docs/config_format.md) through the B200 world and
write the trajectories.

    python -m silk_physics_b200.headless scene.json --out result.npz [--bench]

Scene semantics follow the reference's headless driver
(demo/src/headless.cpp):

* ``global``: dt, max_outer_iteration, max_inner_iteration, acceleration,
  total_steps and the solver tolerances (missing keys keep the
  silk::GlobalConfig defaults);
* ``objects``: ``cloth`` (``cloth`` and ``collision`` configs, optional
  ``pin_selection.bbox`` evaluated after the transform) or ``obstacle``
  (``collision``, optional ``angular_velocity_deg_s``); ``mesh`` is a path
  (relative to the scene file, then to the working directory) to an .obj,
  .off, .ply or .stl triangle mesh;
* ``transform``: x' = translation + Rz Ry Rx (scale * x), with the three
  ``rotation_euler_deg`` values used as radians exactly as the reference's
  transform (demo/src/transform.cpp) uses them, and ``scale`` a number or a
  3-vector;
* an obstacle with an angular velocity is rotated every step, before the
  solver step, by dt x (angular velocity in rad/s) about the mean of its
  transformed vertices, and its new positions are set with
  set_obstacle_position.

Output (unless --bench): an .npz with, per object, ``<name>/positions``
(frames x vertices x 3, float32; frame 0 is the initial state, cloths every
step, rotating obstacles every step, static obstacles only frame 0),
``<name>/faces`` and ``times``.  The Alembic export of the reference is not
provided.
"""
from __future__ import annotations

import argparse
import json
import math
import struct
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import native as N


# ----------------------------------------------------------------------------
# Mesh files
# ----------------------------------------------------------------------------

def _fan(poly):
    return [(poly[0], poly[k], poly[k + 1]) for k in range(1, len(poly) - 1)]


def _load_obj(path: Path):
    verts, faces = [], []
    for lineno, line in enumerate(path.read_text().splitlines(), 1):
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "v":
            if len(parts) < 4:
                raise ValueError(f"line {lineno}: a vertex needs three coordinates")
            verts.append([float(parts[1]), float(parts[2]), float(parts[3])])
        elif parts[0] == "f":
            idx = []
            for tok in parts[1:]:
                i = int(tok.split("/")[0])
                idx.append(i - 1 if i > 0 else len(verts) + i)
            faces.extend(_fan(idx))
    return np.asarray(verts, np.float32), np.asarray(faces, np.int32)


def _load_off(path: Path):
    toks = []
    for line in path.read_text().splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            toks.extend(line.split())
    if not toks[0].upper().endswith("OFF"):
        raise ValueError(f"{path}: not an OFF file")
    toks = toks[1:] if toks[0].upper() == "OFF" else [toks[0][:-3]] + toks[1:]
    nv, nf = int(toks[0]), int(toks[1])
    p = 3
    verts = np.asarray(toks[p:p + 3 * nv], np.float32).reshape(nv, 3)
    p += 3 * nv
    faces = []
    for _ in range(nf):
        k = int(toks[p])
        faces.extend(_fan([int(t) for t in toks[p + 1:p + 1 + k]]))
        p += 1 + k
    return verts, np.asarray(faces, np.int32)


_PLY_TYPES = {"char": "b", "int8": "b", "uchar": "B", "uint8": "B", "short": "h",
              "int16": "h", "ushort": "H", "uint16": "H", "int": "i", "int32": "i",
              "uint": "I", "uint32": "I", "float": "f", "float32": "f", "double": "d",
              "float64": "d"}


def _load_ply(path: Path):
    data = path.read_bytes()
    end = data.index(b"end_header") + len(b"end_header")
    end = data.index(b"\n", end) + 1
    header = data[:end].decode("ascii", "replace").splitlines()
    fmt = "ascii"
    elements = []
    for line in header:
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "format":
            fmt = parts[1]
        elif parts[0] == "element":
            elements.append([parts[1], int(parts[2]), []])
        elif parts[0] == "property":
            elements[-1][2].append(parts[1:])
    body = data[end:]
    verts, faces = [], []
    if fmt == "ascii":
        toks = body.decode("ascii").split()
        p = 0
        for name, count, props in elements:
            for _ in range(count):
                row = []
                for prop in props:
                    if prop[0] == "list":
                        k = int(float(toks[p]))
                        row.append([int(float(t)) for t in toks[p + 1:p + 1 + k]])
                        p += 1 + k
                    else:
                        row.append(float(toks[p]))
                        p += 1
                if name == "vertex":
                    verts.append(_ply_xyz(row, props))
                elif name == "face":
                    faces.extend(_fan(row[0]))
    else:
        endian = "<" if fmt == "binary_little_endian" else ">"
        p = 0
        for name, count, props in elements:
            for _ in range(count):
                row = []
                for prop in props:
                    if prop[0] == "list":
                        ct, it = _PLY_TYPES[prop[1]], _PLY_TYPES[prop[2]]
                        (k,) = struct.unpack_from(endian + ct, body, p)
                        p += struct.calcsize(ct)
                        vals = struct.unpack_from(endian + it * k, body, p)
                        p += struct.calcsize(it) * k
                        row.append(list(vals))
                    else:
                        t = _PLY_TYPES[prop[0]]
                        (v,) = struct.unpack_from(endian + t, body, p)
                        p += struct.calcsize(t)
                        row.append(v)
                if name == "vertex":
                    verts.append(_ply_xyz(row, props))
                elif name == "face":
                    faces.extend(_fan(row[0]))
    return np.asarray(verts, np.float32), np.asarray(faces, np.int32)


def _ply_xyz(row, props):
    names = [pr[-1] for pr in props]
    missing = [a for a in ("x", "y", "z") if a not in names]
    if missing:
        raise ValueError(f"vertex element without propert{'y' if len(missing) == 1 else 'ies'} "
                         f"{', '.join(missing)}")
    return [row[names.index(a)] for a in ("x", "y", "z")]


def _load_stl(path: Path):
    data = path.read_bytes()
    tris = []
    if data[:5] == b"solid" and b"facet" in data[:1024]:
        vs = []
        for line in data.decode("ascii", "replace").splitlines():
            parts = line.split()
            if parts and parts[0] == "vertex":
                vs.append([float(parts[1]), float(parts[2]), float(parts[3])])
        tris = np.asarray(vs, np.float32).reshape(-1, 3, 3)
    else:
        if len(data) < 84:
            raise ValueError("binary STL shorter than its 84-byte header")
        (n,) = struct.unpack_from("<I", data, 80)
        if len(data) < 84 + 50 * n:
            raise ValueError(f"binary STL declares {n} triangles but holds "
                             f"{(len(data) - 84) // 50}")
        rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)),
                                                  ("a", "<u2")]), count=n, offset=84)
        tris = rec["v"].astype(np.float32)
    # Weld identical corners so the cloth is a connected manifold mesh.
    flat = tris.reshape(-1, 3)
    uniq, inv = np.unique(flat, axis=0, return_inverse=True)
    return uniq.astype(np.float32), inv.reshape(-1, 3).astype(np.int32)


def load_mesh(path: Path):
    ext = path.suffix.lower()
    loader = {".obj": _load_obj, ".off": _load_off, ".ply": _load_ply, ".stl": _load_stl}.get(ext)
    if loader is None:
        raise ValueError(f"{path}: unsupported mesh format {ext}")
    try:
        V, F = loader(path)
    except (IndexError, KeyError, struct.error, UnicodeDecodeError, ValueError) as e:
        raise ValueError(f"{path}: malformed {ext[1:].upper()} file ({e})") from e
    if len(V) == 0 or len(F) == 0:
        raise ValueError(f"{path}: empty mesh")
    if F.min() < 0 or F.max() >= len(V):
        raise ValueError(f"{path}: face index out of range ({len(V)} vertices)")
    return V, F


# ----------------------------------------------------------------------------
# Transforms
# ----------------------------------------------------------------------------

def rotation(rx: float, ry: float, rz: float) -> np.ndarray:
    """Rz(rz) Ry(ry) Rx(rx) (angles in radians)."""
    cx, sx, cy, sy, cz, sz = (math.cos(rx), math.sin(rx), math.cos(ry), math.sin(ry),
                              math.cos(rz), math.sin(rz))
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def apply_transform(V: np.ndarray, tr: dict | None) -> np.ndarray:
    if not tr:
        return V.astype(np.float32)
    t = np.asarray(tr.get("translation", [0, 0, 0]), np.float64)
    r = tr.get("rotation_euler_deg", [0, 0, 0])
    s = tr.get("scale", 1.0)
    s = np.full(3, float(s)) if np.isscalar(s) else np.asarray(s, np.float64)
    R = rotation(*[float(a) for a in r])
    out = (V.astype(np.float64) * s) @ R.T + t
    return out.astype(np.float32)


def select_pins(V: np.ndarray, bbox: dict) -> np.ndarray:
    lo = np.minimum(bbox["min"], bbox["max"])
    hi = np.maximum(bbox["min"], bbox["max"])
    inside = np.all((V >= lo) & (V <= hi), axis=1)
    return np.nonzero(inside)[0].astype(np.int32)


# ----------------------------------------------------------------------------
# Scene
# ----------------------------------------------------------------------------

@dataclass
class SceneObject:
    kind: str
    name: str
    verts: np.ndarray
    faces: np.ndarray
    handle: int = 0
    pins: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    omega: np.ndarray = field(default_factory=lambda: np.zeros(3))  # rad/s
    pivot: np.ndarray = field(default_factory=lambda: np.zeros(3))
    frames: list = field(default_factory=list)


def _collision(c: dict | None) -> N.CollisionConfig:
    c = c or {}
    return N.CollisionConfig(is_collision_on=bool(c.get("enabled", True)),
                             is_self_collision_on=bool(c.get("self_collision", True)),
                             group=int(c.get("group", 0)),
                             restitution=float(c.get("restitution", 0.3)),
                             friction=float(c.get("friction", 0.3)))


def _cloth(c: dict | None) -> N.ClothConfig:
    c = c or {}
    d = N.ClothConfig()
    return N.ClothConfig(elastic_stiffness=float(c.get("elastic_stiffness", d.elastic_stiffness)),
                         bending_stiffness=float(c.get("bending_stiffness", d.bending_stiffness)),
                         density=float(c.get("density", d.density)),
                         damping=float(c.get("damping", d.damping)))


def global_config(g: dict) -> N.GlobalConfig:
    d = N.GlobalConfig()
    acc = g.get("acceleration", [d.acceleration_x, d.acceleration_y, d.acceleration_z])
    kw = {k: g[k] for k in ("max_outer_iteration", "max_inner_iteration", "dt",
                            "linear_solver_abs_tol", "linear_solver_rel_tol_min",
                            "linear_solver_rel_tol_max", "initial_linear_rel_tol",
                            "admm_abs_tol", "admm_rel_tol") if k in g}
    return N.GlobalConfig(acceleration_x=float(acc[0]), acceleration_y=float(acc[1]),
                          acceleration_z=float(acc[2]), **kw)


def load_scene(path: str | Path):
    path = Path(path)
    cfg = json.loads(path.read_text())
    objects = []
    for o in cfg.get("objects", []):
        mesh = Path(o["mesh"])
        if not mesh.is_absolute():
            cand = path.parent / mesh
            mesh = cand if cand.exists() else mesh
        if not mesh.exists():
            raise FileNotFoundError(f"{path}: mesh {o['mesh']!r} not found (looked beside the "
                                    f"scene file and in the working directory)")
        V, F = load_mesh(mesh)
        V = apply_transform(V, o.get("transform"))
        kind = o["type"].lower()
        ob = SceneObject(kind, o.get("name", mesh.stem), V, F)
        if kind == "cloth":
            bbox = (o.get("pin_selection") or {}).get("bbox")
            if bbox:
                ob.pins = select_pins(V, bbox)
            ob.cfg = _cloth(o.get("cloth"))
        elif kind == "obstacle":
            w = o.get("angular_velocity_deg_s", [0, 0, 0])
            ob.omega = np.radians(np.asarray(w, np.float64))
            ob.pivot = V.astype(np.float64).mean(0)
        else:
            raise ValueError(f"object {ob.name}: unknown type {o['type']}")
        ob.coll = _collision(o.get("collision"))
        objects.append(ob)
    return cfg.get("global", {}), objects


def write_obj(path: Path, V: np.ndarray, F: np.ndarray) -> None:
    """Triangle mesh as Wavefront OBJ; nine significant digits keep every
    float32 coordinate exact through load_mesh."""
    path.parent.mkdir(parents=True, exist_ok=True)
    lines = [f"v {x:.9g} {y:.9g} {z:.9g}" for x, y, z in np.asarray(V, np.float32).tolist()]
    lines += [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in np.asarray(F, np.int64).tolist()]
    path.write_text("\n".join(lines) + "\n")


def write_scene(directory: str | Path, name: str, scene_text: str,
                meshes: dict) -> Path:
    """Write a scene file and its meshes (mesh path as named in the scene ->
    (vertices, triangles)) under `directory`; returns the scene file's path.
    Meshes are written as OBJ at the named path (whatever its extension), so
    run() loads the same vertices and triangles."""
    d = Path(directory)
    cfg = json.loads(scene_text)
    for o in cfg.get("objects", []):
        V, F = meshes[o["mesh"]]
        obj = Path(o["mesh"]).with_suffix(".obj")
        write_obj(d / obj, V, F)
        o["mesh"] = str(obj)
    path = d / f"{name}.json"
    path.write_text(json.dumps(cfg, indent=2))
    return path


def run(scene: str | Path, out: str | None = None, steps: int | None = None,
        bench: bool = False, options: N.SolverOptions | None = None, log=print):
    """Run a scene; returns (objects with their frames, per-step wall ms)."""
    g, objects = load_scene(scene)
    gcfg = global_config(g)
    w = N.World()
    r = w.init()
    if not r:
        raise RuntimeError(r.to_string())
    r = w.set_global_config(gcfg)
    if not r:
        raise RuntimeError(r.to_string())
    if options is not None:
        w.set_solver_options(options)
    for ob in objects:
        if ob.kind == "cloth":
            r, ob.handle = w.add_cloth(ob.cfg, ob.coll, ob.verts, ob.faces, ob.pins)
        else:
            r, ob.handle = w.add_obstacle(ob.coll, ob.verts, ob.faces)
        if not r:
            raise RuntimeError(f"{ob.name}: {r.to_string()}")
        ob.frames = [ob.verts.copy()]
    total = int(steps if steps is not None else g.get("total_steps", 1))
    dt = gcfg.dt
    times = [0.0]
    wall = []
    buf = {ob.name: np.zeros(ob.verts.size, np.float32) for ob in objects if ob.kind == "cloth"}
    for step in range(total):
        for ob in objects:
            if ob.kind == "obstacle" and np.any(ob.omega != 0.0):
                R = rotation(*(dt * ob.omega))
                V = ((ob.frames[-1].astype(np.float64) - ob.pivot) @ R.T + ob.pivot)
                V = V.astype(np.float32)
                r = w.set_obstacle_position(ob.handle, V.ravel())
                if not r:
                    raise RuntimeError(f"{ob.name}: {r.to_string()}")
                if not bench:
                    ob.frames.append(V)
                else:
                    ob.frames[-1] = V
        t0 = time.perf_counter()
        r = w.solver_step()
        wall.append(1e3 * (time.perf_counter() - t0))
        if not r:
            raise RuntimeError(f"step {step}: {r.to_string()}")
        if not bench:
            times.append((step + 1) * dt)
            for ob in objects:
                if ob.kind == "cloth":
                    w.get_cloth_position(ob.handle, buf[ob.name])
                    ob.frames.append(buf[ob.name].reshape(-1, 3).copy())
        if log:
            log(f"step {step}: {wall[-1]:.1f} ms")
    if out and not bench:
        arrays = {"times": np.asarray(times, np.float32)}
        for ob in objects:
            arrays[f"{ob.name}/positions"] = np.stack(ob.frames)
            arrays[f"{ob.name}/faces"] = ob.faces
        np.savez(out, **arrays)
    return objects, wall


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="Run a JSON scene headless on the GPU.")
    ap.add_argument("scene")
    ap.add_argument("--out", default="result.npz")
    ap.add_argument("--steps", type=int, default=None, help="override global.total_steps")
    ap.add_argument("--bench", action="store_true", help="time the steps, write nothing")
    a = ap.parse_args(argv)
    _, wall = run(a.scene, a.out, a.steps, a.bench)
    n = len(wall)
    print(f"{n} steps, {sum(wall) / max(n, 1):.2f} ms per step"
          + ("" if a.bench else f", trajectories written to {a.out}"), file=sys.stderr)


if __name__ == "__main__":
    main()
