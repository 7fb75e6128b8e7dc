"""Synthetic scenes of the benchmark configurations.

* ``grid_sheet``: square cloth as a regular s x s vertex grid with alternating
  diagonals, in the XY plane (the "6K cloth" of the reference README is
  model/dense_sheet.obj; these sheets stand in for it with seeded shapes).
* ``icosphere``: subdivided icosahedron (subdivision 4 = 2,562 vertices,
  5,120 triangles).
"""
from __future__ import annotations

import numpy as np


def grid_sheet(side_count: int, side: float = 1.0, z: float = 1.0,
               jitter: float = 0.0, seed: int = 0, center=(0.0, 0.0)):
    """Return (verts[float32, n x 3], faces[int32, m x 3])."""
    s = side_count
    xs = np.linspace(-side / 2, side / 2, s, dtype=np.float64)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    V = np.stack([X.ravel() + center[0], Y.ravel() + center[1],
                  np.full(s * s, z)], axis=1)
    if jitter > 0:
        V += np.random.default_rng(seed).normal(0.0, jitter, V.shape)
    idx = np.arange(s * s).reshape(s, s)
    faces = []
    for j in range(s - 1):
        for i in range(s - 1):
            a, b, c, d = idx[j, i], idx[j, i + 1], idx[j + 1, i], idx[j + 1, i + 1]
            if (i + j) % 2 == 0:
                faces += [(a, b, d), (a, d, c)]
            else:
                faces += [(a, b, c), (b, d, c)]
    return V.astype(np.float32), np.asarray(faces, np.int32)


def top_corner_pins(side_count: int) -> np.ndarray:
    """Indices of the two corners at maximum y."""
    s = side_count
    return np.asarray([(s - 1) * s, s * s - 1], np.int32)


def icosphere(subdivisions: int = 4, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    t = (1.0 + 5 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    V = [np.asarray(v, np.float64) / np.linalg.norm(v) for v in V]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9),
         (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2),
         (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                cache[key] = len(V) - 1
            return cache[key]

        nf = []
        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = nf
    Vn = np.asarray(V) * radius + np.asarray(center)
    return Vn.astype(np.float32), np.asarray(F, np.int32)


# Benchmark configurations (sizes and physical parameters).
CONFIGS = {
    "c1_sheet32_pinned": dict(side_count=32, side=1.0, z=1.0, jitter=0.0, pins=True,
                              sphere=None, steps=100, max_inner=10),
    "c2_sheet80_sphere": dict(side_count=80, side=1.0, z=1.0, jitter=1e-4, pins=False,
                              sphere=0.3, steps=300, max_inner=100),
    "c3_sheet316_sphere": dict(side_count=316, side=2.0, z=1.0, jitter=1e-4, pins=False,
                               sphere=0.6, steps=200, max_inner=100),
}


def c2_scene(seed: int = 1236):
    """6.4K-vertex sheet on a sphere: 80 x 80 grid (12,482 triangles), side
    1 m, jitter N(0, 1e-4) m, at z = 1 above an icosphere of subdivision 4
    and radius 0.3 m at the origin.  Returns (V, F, SV, SF)."""
    V, F = grid_sheet(80, side=1.0, z=1.0, jitter=1e-4, seed=seed)
    SV, SF = icosphere(4, radius=0.3)
    return V, F, SV, SF


def c3_scene(seed: int = 1237):
    """100K-vertex drape: 316 x 316 grid (99,856 vertices, 198,450
    triangles), side 2 m, jitter N(0, 1e-4) m, at z = 0.7, 0.1 m above an
    icosphere of subdivision 4 and radius 0.6 m at the origin.  Returns
    (V, F, SV, SF)."""
    V, F = grid_sheet(316, side=2.0, z=0.7, jitter=1e-4, seed=seed)
    SV, SF = icosphere(4, radius=0.6)
    return V, F, SV, SF


def free_fall_state(V, steps: int, dt: float = 1.0 / 60.0, g: float = -9.81,
                    damping: float = 0.01):
    """Positions and velocities of an unpinned, unstressed sheet after
    `steps` steps of free fall from rest (each step damps the velocity by
    1 - damping, adds g dt and moves by v dt, main_loop.cu:24-120).  Returns
    float32 (x, v) in mesh order."""
    vz = 0.0
    dz = 0.0
    for _ in range(steps):
        vz = (1.0 - damping) * vz + g * dt
        dz += vz * dt
    x = np.asarray(V, np.float64).copy()
    x[:, 2] += dz
    v = np.zeros_like(x)
    v[:, 2] = vz
    return x.astype(np.float32), v.astype(np.float32)

