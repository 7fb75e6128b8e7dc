"""Learned CG warm start: data collection from the solver, training on the
GPU and model files.

The model (see ``silk_set_warm_start_model`` in include/silk_b200.h) is a
per-vertex MLP 13 -> 64 -> 64 -> 64 -> 3 whose output, scaled by the step scale
dt^2 |g| and a per-channel output scale, is added to the inertial prediction
to form a candidate start for the first CG solve of each outer iteration.
Samples are recorded by the solver itself (solver option capture_samples);
training runs the library's own GPU kernels (tensor-core forward, FP32
backward, Adam) through ``native.mlp_train``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import native as N
from . import scenes as S

N_IN = 13
K_IN = 16
H = 64
K_OUT = 8
# Offsets of the parameter vector (FP32), in the order of the C header.
_SHAPES = [("W1", (K_IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
           ("W3", (H, H)), ("b3", (H,)), ("W4", (H, K_OUT)), ("b4", (K_OUT,)),
           ("feat_mean", (K_IN,)), ("feat_std", (K_IN,)), ("out_scale", (K_OUT,))]
OFFSETS = {}
_o = 0
for _name, _shp in _SHAPES:
    OFFSETS[_name] = (_o, _shp)
    _o += int(np.prod(_shp))
N_PARAMS = _o
assert N_PARAMS == N.MLP_PARAMS


def put(params: np.ndarray, name: str, value) -> None:
    o, shp = OFFSETS[name]
    params[o:o + int(np.prod(shp))] = np.asarray(value, np.float32).ravel()


def get(params: np.ndarray, name: str) -> np.ndarray:
    o, shp = OFFSETS[name]
    return params[o:o + int(np.prod(shp))].reshape(shp)


def initial_params(feat_mean, feat_std, out_scale, seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases and the given statistics."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    w1 = rng.normal(0, math.sqrt(2.0 / N_IN), (K_IN, H))
    w1[N_IN:] = 0.0
    put(p, "W1", w1)
    put(p, "W2", rng.normal(0, math.sqrt(2.0 / H), (H, H)))
    put(p, "W3", rng.normal(0, math.sqrt(2.0 / H), (H, H)))
    w4 = rng.normal(0, math.sqrt(1.0 / H), (H, K_OUT)) * 0.1
    w4[:, 3:] = 0.0
    put(p, "W4", w4)
    put(p, "feat_mean", feat_mean)
    put(p, "feat_std", feat_std)
    put(p, "out_scale", out_scale)
    return p


@dataclass
class SampleSet:
    features: list = field(default_factory=list)
    targets: list = field(default_factory=list)

    def add(self, f: np.ndarray, t: np.ndarray, keep: int, rng) -> None:
        if keep < len(f):
            idx = rng.choice(len(f), keep, replace=False)
            f, t = f[idx], t[idx]
        self.features.append(f)
        self.targets.append(t)

    def arrays(self) -> tuple[np.ndarray, np.ndarray]:
        return np.concatenate(self.features), np.concatenate(self.targets)


def _world(V, F, pins, SV=None, SF=None, inner=100, capture=True, tol=1e-5):
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81, max_inner_iteration=inner))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=tol,
                                                capture_samples=capture))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, pins)
    assert r, r.to_string()
    if SV is not None:
        r, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
        assert r
    return w, h


def collect(scenes, steps: int, keep_per_step: int = 4096, seed: int = 0,
            samples: SampleSet | None = None, budget_s: float = 20.0) -> SampleSet:
    """Run each scene (V, F, pins, SV, SF, inner) for up to `steps` steps (and
    at most budget_s seconds) and keep up to keep_per_step vertex samples of
    every step that recorded some."""
    import time

    rng = np.random.default_rng(seed)
    samples = samples or SampleSet()
    for V, F, pins, SV, SF, inner in scenes:
        w, h = _world(V, F, pins, SV, SF, inner)
        t0 = time.time()
        for _ in range(steps):
            if time.time() - t0 > budget_s:
                break
            r = w.solver_step()
            if not r:
                break
            got = w.warm_start_samples(h, len(V))
            if got is not None:
                f, t = got
                samples.add(f, t, keep_per_step, rng)
    return samples


def training_scenes(rng, count: int, sides=(40, 120), radii=(0.2, 0.8)):
    """Sheets of random side counts over spheres of random radii, plus the
    pinned-corner sheet: the mix of the warm-start training set."""
    out = []
    for k in range(count):
        s = int(round(math.exp(rng.uniform(math.log(sides[0]), math.log(sides[1])))))
        r = float(rng.uniform(*radii))
        V, F = S.grid_sheet(s, side=1.0, z=r + 0.1, jitter=1e-4, seed=int(rng.integers(1 << 30)))
        SV, SF = S.icosphere(3, r)
        pins = S.top_corner_pins(s) if k % 3 == 0 else np.zeros(0, np.int32)
        out.append((V, F, pins, SV if k % 3 else None, SF if k % 3 else None, 100))
    return out


def statistics(features: np.ndarray, targets: np.ndarray):
    """Feature standardisation and per-channel output scale."""
    mean = np.zeros(K_IN, np.float32)
    std = np.ones(K_IN, np.float32)
    mean[:N_IN] = features[:, :N_IN].mean(0)
    std[:N_IN] = np.maximum(features[:, :N_IN].std(0), 1e-3)
    out = np.ones(K_OUT, np.float32)
    out[:3] = np.maximum(targets[:, :3].std(0), 1e-6)
    return mean, std, out


def normalised_targets(targets: np.ndarray, out_scale: np.ndarray) -> np.ndarray:
    t = np.zeros((len(targets), 4), np.float32)
    t[:, :3] = targets[:, :3] / out_scale[:3]
    return t


def train(features: np.ndarray, targets: np.ndarray, steps: int = 2000, batch: int = 65536,
          lr: float = 2e-3, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Fit the model on (features n x 16, raw targets n x 4) on the GPU;
    returns (parameters, loss per step)."""
    mean, std, out = statistics(features, targets)
    p0 = initial_params(mean, std, out, seed)
    return N.mlp_train(p0, features, normalised_targets(targets, out), steps, batch, lr, seed)


def save(path: str, params: np.ndarray) -> None:
    np.save(path, np.asarray(params, np.float32))


def load(path: str) -> np.ndarray:
    p = np.load(path).astype(np.float32)
    if p.size != N_PARAMS:
        raise ValueError(f"{path}: expected {N_PARAMS} parameters, got {p.size}")
    return p


def main(argv=None) -> None:
    """Generate solver samples, train on the GPU and save the model:

    python -m silk_physics_b200.learned --out silk_physics_b200/models/warm_start.npy
    """
    import argparse
    import time

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--out", required=True)
    ap.add_argument("--scenes", type=int, default=12)
    ap.add_argument("--steps", type=int, default=40, help="solver steps per scene")
    ap.add_argument("--keep", type=int, default=4096, help="vertex samples kept per step")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    t0 = time.time()
    scenes = training_scenes(rng, a.scenes)
    samples = collect(scenes, a.steps, a.keep, a.seed)
    f, t = samples.arrays()
    t1 = time.time()
    p, hist = train(f, t, a.train_steps, a.batch, a.lr, a.seed)
    t2 = time.time()
    save(a.out, p)
    print(f"{len(f)} samples from {a.scenes} scenes x {a.steps} steps in {t1 - t0:.1f} s; "
          f"trained {a.train_steps} steps in {t2 - t1:.1f} s; loss {hist[0]:.4f} -> "
          f"{hist[-1]:.4f}; saved {a.out}")


if __name__ == "__main__":
    main()
