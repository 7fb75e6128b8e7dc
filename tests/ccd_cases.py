"""Seeded CCD query families shared by the CCD parity tests.

Each query is 24 floats: four points at t0, then the same four at t1
(vertex-face: the vertex first, then the triangle's corners; edge-edge: the
first edge's ends, then the second's)."""
import numpy as np

ERR = {True: 4.053116e-06, False: 3.814698e-06}  # interval_root_finder.cpp:516-517


def random_queries(rng, n, vf):
    """Crossing motions of unit-scale primitives (a mix of hits and misses)."""
    base = rng.uniform(-1, 1, (n, 4, 3)).astype(np.float32)
    if vf:
        base[:, 1:, 2] = 0.0
        base[:, 0, 2] = rng.uniform(0.001, 0.2, n)
    motion = rng.normal(0, 0.4, (n, 4, 3)).astype(np.float32)
    motion[:, 0, 2] -= rng.uniform(0, 0.6, n)
    x = np.concatenate([base, base + motion], axis=1)
    return x.reshape(n, 24).astype(np.float32)


def near_contact_queries(rng, n, vf, ms=1e-3):
    """Primitives that start within about two minimum separations of each
    other and approach: many hits at t = 0, which exercise the refined
    separation retry (no_zero_toi, ccd.cpp:150-180)."""
    base = rng.uniform(-1, 1, (n, 4, 3)).astype(np.float32)
    if vf:
        base[:, 1:, 2] = 0.0
        base[:, 0, :2] = rng.uniform(-0.2, 0.2, (n, 2))
        base[:, 1] = (-1.0, -1.0, 0.0)
        base[:, 2] = (1.0, -1.0, 0.0)
        base[:, 3] = (0.0, 1.0, 0.0)
        base[:, 0, 2] = rng.uniform(0.0, 2.0 * ms, n)
    else:
        base[:, 0] = (-1.0, 0.0, 0.0)
        base[:, 1] = (1.0, 0.0, 0.0)
        base[:, 2, :2] = (0.0, -1.0)
        base[:, 3, :2] = (0.0, 1.0)
        base[:, 2:, 2] = rng.uniform(0.0, 2.0 * ms, n)[:, None]
    motion = rng.normal(0, 0.05, (n, 4, 3)).astype(np.float32)
    motion[:, 0, 2] -= rng.uniform(0, 0.2, n)
    x = np.concatenate([base, base + motion], axis=1)
    return x.reshape(n, 24).astype(np.float32)


def query_set(vf, n_random=1500, n_near=500, seed=0):
    """(x, ms): random and near-contact queries with separations 0, 1e-4 and
    1e-3."""
    rng = np.random.default_rng((1000 if vf else 2000) + seed)
    x = np.concatenate([random_queries(rng, n_random, vf), near_contact_queries(rng, n_near, vf)])
    ms = np.concatenate([rng.choice([0.0, 1e-4, 1e-3], n_random),
                         rng.choice([1e-4, 1e-3], n_near)]).astype(np.float32)
    return x, ms
