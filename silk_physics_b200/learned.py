"""Learned CG warm start: data collection from the solver, training on the
GPU and model files.

Two per-vertex MLPs 13 -> 64 -> 64 -> 64 -> 3 (see ``silk_set_warm_start_model``
in include/silk_b200.h):

* the first-solve model: its output, scaled by the step scale dt^2 |g| and a
  per-channel output scale, is added to the inertial prediction to form a
  candidate start for the first CG solve of each outer iteration;
* the iterate model: from the last three ADMM iterates it predicts the next
  one, offered as the start of every later CG solve of the ADMM solve.

Samples are recorded by the solver itself (solver option capture_samples);
training runs the library's own GPU kernels (tensor-core forward, FP32
backward, Adam) through ``native.mlp_train``.  A model file holds the
first-solve model, optionally followed by the iterate model.
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


def _world(V, F, pins, SV=None, SF=None, inner=100, capture=1, tol=1e-5):
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81, max_inner_iteration=inner))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=tol,
                                                capture_samples=int(capture)))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, pins)
    assert r, r.to_string()
    if SV is not None:
        r, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
        assert r
    return w, h


@dataclass
class Scene:
    """A training scene: sheet, pins, optional sphere, ADMM iteration cap and
    the state the sheet starts from (None: at rest)."""
    V: np.ndarray
    F: np.ndarray
    pins: np.ndarray
    SV: np.ndarray | None = None
    SF: np.ndarray | None = None
    inner: int = 100
    x0: np.ndarray | None = None
    v0: np.ndarray | None = None


def collect_both(scenes, steps: int, keep_first: int = 4096, keep_iter: int = 16384,
                 seed: int = 0, budget_s: float = 60.0, log=print):
    """Run each scene for up to `steps` steps (at most budget_s seconds each)
    recording both sample sets; keeps up to keep_first first-solve and
    keep_iter iterate samples of every step.  Returns (first-solve samples,
    iterate samples, solver steps run)."""
    import time

    rng = np.random.default_rng(seed)
    first, iterate = SampleSet(), SampleSet()
    nsteps = 0
    for k, sc in enumerate(scenes):
        w, h = _world(sc.V, sc.F, sc.pins, sc.SV, sc.SF, sc.inner, capture=3)
        if sc.x0 is not None:
            assert w.set_cloth_state(h, sc.x0, sc.v0)
        t0 = time.time()
        for _ in range(steps):
            if time.time() - t0 > budget_s:
                break
            r = w.solver_step()
            if not r:
                break
            nsteps += 1
            got = w.warm_start_samples(h, len(sc.V))
            if got is not None:
                first.add(got[0], got[1], keep_first, rng)
            f, t = w.iterate_samples()
            if len(f):
                iterate.add(f, t, keep_iter, rng)
        if log:
            log(f"scene {k}: {len(sc.V)} vertices, {nsteps} steps so far, "
                f"{sum(len(a) for a in iterate.features)} iterate samples")
    return first, iterate, nsteps


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


def training_mix(rng, count: int, sides=(40, 200), radii=(0.2, 0.8)) -> list:
    """The training mix: the 32 x 32 pinned sheet of config 1 (10 ADMM
    iterations), the 80 x 80 sheet on the r = 0.3 m sphere of config 2, and
    sheets of log-uniform side counts in `sides` over spheres of radii
    uniform in `radii`, every sphere scene starting from its free-fall state
    a step or two before contact so that every step collected is a contact
    step."""
    out = [Scene(*S.grid_sheet(32, jitter=1e-4, seed=int(rng.integers(1 << 30))),
                 S.top_corner_pins(32), inner=10)]
    V, F, SV, SF = S.c2_scene(seed=int(rng.integers(1 << 30)))
    x0, v0 = S.free_fall_state(V, 24)
    out.append(Scene(V, F, np.zeros(0, np.int32), SV, SF, 100, x0, v0))
    for _ in range(max(count - 2, 0)):
        s = int(round(math.exp(rng.uniform(math.log(sides[0]), math.log(sides[1])))))
        r = float(rng.uniform(*radii))
        side = float(rng.uniform(0.8, 2.0))
        V, F = S.grid_sheet(s, side=side, z=r + 0.1, jitter=1e-4, seed=int(rng.integers(1 << 30)))
        SV, SF = S.icosphere(4, r)
        x0, v0 = S.free_fall_state(V, 7)
        out.append(Scene(V, F, np.zeros(0, np.int32), SV, SF, 100, x0, v0))
    return out


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
    """A model file: the first-solve model (N_PARAMS floats), optionally
    followed by the iterate model (2 N_PARAMS floats in all)."""
    p = np.load(path).astype(np.float32).ravel()
    if p.size not in (N_PARAMS, 2 * N_PARAMS):
        raise ValueError(f"{path}: expected {N_PARAMS} or {2 * N_PARAMS} parameters, got {p.size}")
    return p


def main(argv=None) -> None:
    """Generate solver samples on the training mix, train both models on the
    GPU and save them:

    python -m silk_physics_b200.learned --out silk_physics_b200/models/warm_start.npy
    """
    import argparse
    import time

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--out", required=True)
    ap.add_argument("--scenes", type=int, default=24)
    ap.add_argument("--steps", type=int, default=6, help="solver steps per scene")
    ap.add_argument("--keep", type=int, default=4096, help="first-solve samples kept per step")
    ap.add_argument("--keep-iter", type=int, default=16384,
                    help="iterate samples kept per step")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    t0 = time.time()
    scenes = training_mix(rng, a.scenes)
    first, iterate, nsteps = collect_both(scenes, a.steps, a.keep, a.keep_iter, a.seed)
    f1, t1_ = first.arrays()
    f2, t2_ = iterate.arrays()
    t1 = time.time()
    p1, h1 = train(f1, t1_, a.train_steps, a.batch, a.lr, a.seed)
    p2, h2 = train(f2, t2_, a.train_steps, a.batch, a.lr, a.seed + 1)
    t2 = time.time()
    save(a.out, np.concatenate([p1, p2]))
    print(f"{nsteps} solver steps of {len(scenes)} scenes in {t1 - t0:.1f} s: "
          f"{len(f1)} first-solve and {len(f2)} iterate samples; trained {a.train_steps} "
          f"steps each in {t2 - t1:.1f} s; loss first-solve {h1[0]:.4f} -> {h1[-1]:.4f}, "
          f"iterate {h2[0]:.4f} -> {h2[-1]:.4f}; saved {a.out}")


if __name__ == "__main__":
    main()
