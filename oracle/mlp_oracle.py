"""CPU restatement (FP64, numpy) of the learned CG warm start.

TEST INFRASTRUCTURE: used only by tests/ to check the GPU kernels of
silk_physics_b200/csrc/learned.cu (forward, gradients, training step); never
imported by the product path.

The learned warm start has no counterpart in the reference (it predicts the
initial guess of the first CG solve of an outer iteration,
mas_cg_solver.cu:193-311 starts from the current state).  Model, shared with
the GPU kernels:

* 13 features per vertex: inertial prediction minus start position (3), last
  displacement (3), the displacement before (3), 1-ring mean of the last
  displacement (3), pin flag (1); displacement features are divided by the
  step scale sigma = dt^2 |g| (1e-12 floor), then standardised with the
  model's mean / std (inputs padded to 16 with zeros);
* MLP 16 -> 64 -> 64 -> 64 -> 8 (3 outputs used), exact-erf GELU on the hidden
  layers; weights and every layer input are rounded to BF16 (round to nearest
  even) before the product, accumulation is FP32 on the GPU and FP64 here;
* prediction = start guess y + sigma * out_scale * output;
* loss = mean over samples and the 3 outputs of (output - target_hat)^2 with
  target_hat = (target / sigma) / out_scale;
* backward treats the BF16 rounding as the identity (straight-through) and
  uses the rounded weights and inputs in the products.
"""
from __future__ import annotations

import math

import numpy as np

N_IN = 13
K_IN = 16
H = 64
N_OUT = 3
K_OUT = 8

# Parameter vector layout (FP32 on the GPU).
SHAPES = [("W1", (K_IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
          ("W3", (H, H)), ("b3", (H,)), ("W4", (H, K_OUT)), ("b4", (K_OUT,)),
          ("feat_mean", (K_IN,)), ("feat_std", (K_IN,)), ("out_scale", (K_OUT,))]
N_TRAINABLE = 8  # the first 8 entries are learned; the rest are statistics


def offsets():
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = (o, shp)
        o += n
    return out, o


OFFSETS, N_PARAMS = offsets()
N_TRAIN_PARAMS = OFFSETS["feat_mean"][0]


def unpack(p):
    return {k: np.asarray(p[o:o + int(np.prod(s))], np.float64).reshape(s)
            for k, (o, s) in OFFSETS.items()}


# Finite-difference self-checks turn the rounding off (the rounded model is
# piecewise constant in its inputs); the GPU comparison keeps it on.
ROUND = True


def bf16(x):
    """Round float values to BF16 (nearest even), returned as float64."""
    if not ROUND:
        return np.asarray(x, np.float64)
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(a)
    if nan.any():
        out[nan] = np.nan
    return out


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(
        2.0 * math.pi)


def normalise(features, P):
    """features: (n, 13) already divided by sigma where applicable."""
    f = np.zeros((len(features), K_IN))
    f[:, :N_IN] = features
    return (f - P["feat_mean"]) / P["feat_std"]


def forward(P, xn):
    """xn: (n, 16) normalised inputs.  Returns output (n, 8) and the cache."""
    cache = []
    h = xn
    for i in range(1, 4):
        a = bf16(h)
        z = a @ bf16(P[f"W{i}"]) + P[f"b{i}"]
        cache.append((a, z))
        h = gelu(z)
    a = bf16(h)
    out = a @ bf16(P["W4"]) + P["b4"]
    cache.append((a, None))
    return out, cache


def loss_and_grad(p, xn, t_hat):
    """Mean squared error over samples and the 3 outputs; gradient w.r.t. the
    trainable part of the parameter vector (same layout, statistics zero)."""
    P = unpack(p)
    out, cache = forward(P, xn)
    n = len(xn)
    d = np.zeros_like(out)
    d[:, :N_OUT] = out[:, :N_OUT] - t_hat
    loss = float((d[:, :N_OUT] ** 2).sum() / (n * N_OUT))
    g = {}
    delta = 2.0 * d / (n * N_OUT)
    a4, _ = cache[3]
    g["W4"] = a4.T @ delta
    g["b4"] = delta.sum(0)
    back = delta @ bf16(P["W4"]).T
    for i in (3, 2, 1):
        a, z = cache[i - 1]
        delta = back * gelu_grad(z)
        g[f"W{i}"] = a.T @ delta
        g[f"b{i}"] = delta.sum(0)
        back = delta @ bf16(P[f"W{i}"]).T
    grad = np.zeros(N_PARAMS)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        o, s = OFFSETS[k]
        grad[o:o + int(np.prod(s))] = g[k].ravel()
    # Padded output columns carry no loss.
    o, _ = OFFSETS["W4"]
    W4g = grad[o:o + H * K_OUT].reshape(H, K_OUT)
    W4g[:, N_OUT:] = 0.0
    o, _ = OFFSETS["b4"]
    grad[o + N_OUT:o + K_OUT] = 0.0
    return loss, grad


def init_params(seed=0, feat_mean=None, feat_std=None, out_scale=None):
    """He-style initial weights (the GPU trainer starts from the same)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)

    def put(name, v):
        o, s = OFFSETS[name]
        p[o:o + int(np.prod(s))] = np.asarray(v, np.float32).ravel()

    put("W1", rng.normal(0, math.sqrt(2.0 / N_IN), (K_IN, H)) * (np.arange(K_IN) < N_IN)[:, None])
    put("W2", rng.normal(0, math.sqrt(2.0 / H), (H, H)))
    put("W3", rng.normal(0, math.sqrt(2.0 / H), (H, H)))
    w4 = rng.normal(0, math.sqrt(1.0 / H), (H, K_OUT))
    w4[:, N_OUT:] = 0.0
    put("W4", w4)
    put("feat_mean", np.zeros(K_IN) if feat_mean is None else feat_mean)
    put("feat_std", np.ones(K_IN) if feat_std is None else feat_std)
    put("out_scale", np.ones(K_OUT) if out_scale is None else out_scale)
    return p


def adam_step(p, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trainable part (FP64 restatement of the GPU step)."""
    n = N_TRAIN_PARAMS
    g = grad[:n]
    m[:n] = b1 * m[:n] + (1 - b1) * g
    v[:n] = b2 * v[:n] + (1 - b2) * g * g
    mh = m[:n] / (1 - b1 ** step)
    vh = v[:n] / (1 - b2 ** step)
    p = np.array(p, np.float64)
    p[:n] -= lr * mh / (np.sqrt(vh) + eps)
    return p


def features(x0, x1, x2, y, pins, ring_off, ring, sigma):
    """Per-vertex features from the start position x0, the two previous step
    positions x1, x2, the inertial prediction y (all (n, 3)), pin flags and the
    1-ring CSR; displacement features divided by sigma."""
    n = len(x0)
    d1 = x0 - x1
    f = np.zeros((n, N_IN))
    f[:, 0:3] = (y - x0) / sigma
    f[:, 3:6] = d1 / sigma
    f[:, 6:9] = (x1 - x2) / sigma
    for v in range(n):
        nb = ring[ring_off[v]:ring_off[v + 1]]
        if len(nb):
            f[v, 9:12] = d1[nb].mean(0) / sigma
    f[:, 12] = pins
    return f
