"""Learned CG warm start: the GPU MLP kernels against the FP64 oracle
(forward, loss gradient, Adam step), training on the GPU, and the solver
integration (samples, learned start taken or refused, what it gains)."""
import sys
from pathlib import Path

import numpy as np
import pytest

from silk_physics_b200 import learned as L
from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as M  # noqa: E402

# BF16 layer inputs: an FP32 pre-activation that lands next to a BF16
# rounding boundary can round the other way than the FP64 restatement, so
# outputs and gradients are compared in norm with these relative tolerances.
FWD_TOL = 2e-2
GRAD_TOL = 3e-2


def _random_case(n, seed):
    rng = np.random.default_rng(seed)
    feats = np.zeros((n, 16), np.float32)
    feats[:, :13] = rng.normal(0, 2.0, (n, 13))
    feats[:, 12] = rng.integers(0, 2, n)
    mean = np.zeros(16, np.float32)
    std = np.ones(16, np.float32)
    mean[:13] = rng.normal(0, 0.5, 13)
    std[:13] = rng.uniform(0.5, 2.0, 13)
    p = M.init_params(seed, mean, std, np.array([1.5, 0.7, 2.0, 1, 1, 1, 1, 1], np.float32))
    o, _ = M.OFFSETS["b1"]
    p[o:o + 64] = rng.normal(0, 0.1, 64)
    t = np.zeros((n, 4), np.float32)
    t[:, :3] = rng.normal(0, 1.0, (n, 3))
    return p, feats, t


def test_layouts_agree():
    assert L.N_PARAMS == M.N_PARAMS == N.MLP_PARAMS
    for k, (o, s) in M.OFFSETS.items():
        assert L.OFFSETS[k] == (o, s)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = M.init_params(2).astype(np.float64)
    xn = rng.normal(size=(40, 16))
    xn[:, 13:] = 0
    t = rng.normal(size=(40, 3))
    M.ROUND = False
    try:
        _, g = M.loss_and_grad(p, xn, t)
        for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
            o, s = M.OFFSETS[name]
            for j in rng.choice(int(np.prod(s)), 4, replace=False):
                if name == "W4" and j % 8 >= 3:
                    continue
                if name == "W1" and j // 64 >= 13:
                    continue
                e = 1e-6
                pp, pm = p.copy(), p.copy()
                pp[o + j] += e
                pm[o + j] -= e
                fd = (M.loss_and_grad(pp, xn, t)[0] - M.loss_and_grad(pm, xn, t)[0]) / (2 * e)
                assert abs(fd - g[o + j]) <= 1e-5 * max(1.0, abs(fd)), (name, j)
    finally:
        M.ROUND = True


@pytest.mark.gpu
def test_forward_matches_oracle():
    p, f, _ = _random_case(1000, 1)
    out = N.mlp_forward(p, f)
    P = M.unpack(p)
    ref, _ = M.forward(P, (f.astype(np.float64) - P["feat_mean"]) / P["feat_std"])
    ref = ref[:, :3]
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    print(f"forward: relative error {err:.2e}, max abs {np.abs(out - ref).max():.2e}")
    assert err < FWD_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 129, 200_003])
def test_forward_tiles_match_oracle(n):
    """The inference forward (tcgen05.mma, 128-sample tiles, accumulators in
    tensor memory; persistent CTAs take several tiles once n passes 4 tiles
    per SM): every size against the oracle, and a sample's output does not
    depend on the batch it is in (tiles are independent, so the first rows
    of a larger batch are bit-identical to the same rows alone)."""
    p, f, _ = _random_case(n, 5)
    out = N.mlp_forward(p, f)
    P = M.unpack(p)
    ref, _ = M.forward(P, (f.astype(np.float64) - P["feat_mean"]) / P["feat_std"])
    ref = ref[:, :3]
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    print(f"n={n}: relative error {err:.2e}, max abs {np.abs(out - ref).max():.2e}")
    assert np.isfinite(out).all()
    assert err < FWD_TOL
    head = min(n, 100)
    np.testing.assert_array_equal(N.mlp_forward(p, f[:head]), out[:head])


@pytest.mark.gpu
def test_loss_gradient_matches_oracle():
    p, f, t = _random_case(3000, 2)
    loss, grad = N.mlp_loss_grad(p, f, t)
    P = M.unpack(p)
    xn = (f.astype(np.float64) - P["feat_mean"]) / P["feat_std"]
    rloss, rgrad = M.loss_and_grad(p.astype(np.float64), xn, t[:, :3].astype(np.float64))
    print(f"loss gpu {loss:.6f} oracle {rloss:.6f}")
    assert abs(loss - rloss) <= FWD_TOL * rloss
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        o, s = M.OFFSETS[name]
        n = int(np.prod(s))
        g, r = grad[o:o + n], rgrad[o:o + n]
        err = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-12)
        print(f"{name}: relative gradient error {err:.2e}")
        assert err < GRAD_TOL, name
    assert np.all(grad[M.N_TRAIN_PARAMS:] == 0)


@pytest.mark.gpu
def test_adam_step_matches_oracle():
    p, f, t = _random_case(2000, 4)
    p1, _ = N.mlp_train(p, f, t, steps=1, batch=0, lr=1e-3)
    _, g = N.mlp_loss_grad(p, f, t)
    m = np.zeros(M.N_PARAMS)
    v = np.zeros(M.N_PARAMS)
    ref = M.adam_step(p, g.astype(np.float64), m, v, 1, 1e-3)
    np.testing.assert_allclose(p1, ref, rtol=0, atol=2e-6)
    assert np.all(p1[M.N_TRAIN_PARAMS:] == p[M.N_TRAIN_PARAMS:])


@pytest.mark.gpu
def test_training_reduces_loss():
    rng = np.random.default_rng(5)
    n = 20000
    f = np.zeros((n, 16), np.float32)
    f[:, :13] = rng.normal(0, 1.0, (n, 13))
    t = np.zeros((n, 4), np.float32)
    t[:, 0] = np.tanh(f[:, 0] - 0.5 * f[:, 3])
    t[:, 1] = f[:, 1] * f[:, 4] * 0.5
    t[:, 2] = np.sin(f[:, 2]) + 0.3 * f[:, 9]
    p, hist = L.train(f, t, steps=400, batch=4096, lr=3e-3)
    print(f"loss {hist[0]:.4f} -> {hist[-1]:.4f}")
    assert hist[-1] < 0.2 * hist[0]


def _pinned_sheet(s, seed):
    V, F = S.grid_sheet(s, jitter=1e-4, seed=seed)
    return V, F, S.top_corner_pins(s)


def _run(V, F, P, steps, params=None, learned=False, capture=False):
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81, max_inner_iteration=10,
                                              admm_abs_tol=0.0, admm_rel_tol=0.0))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5,
                                                learned_warm_start=learned,
                                                capture_samples=capture))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(is_collision_on=False,
                                                          is_self_collision_on=False),
                       V, F, P)
    assert r
    if params is not None:
        assert w.set_warm_start_model(params)
    first, taken, samples = 0, 0, []
    x = np.zeros(V.size, np.float32)
    for _ in range(steps):
        assert w.solver_step(), w
        st = w.step_stats()
        first += st.cg_first_solve_iterations
        taken += st.learned_starts
        if capture:
            got = w.warm_start_samples(h, len(V))
            assert got is not None
            samples.append(got)
    w.get_cloth_position(h, x)
    return first, taken, x.reshape(-1, 3), samples


@pytest.mark.gpu
def test_learned_warm_start_in_the_solver():
    """Train on samples the solver records from pinned swinging sheets, then
    run a held-out sheet: the CG starts from the residual-minimising blend of
    the plain and the learned start where that lowers the residual, positions
    stay within the CG tolerance's reach of the plain run, and a model that
    predicts no correction is never taken (bit-identical to the plain run)."""
    samples = L.SampleSet()
    rng = np.random.default_rng(0)
    for s, seed in ((24, 1), (32, 2), (40, 3)):
        V, F, P = _pinned_sheet(s, seed)
        _, _, _, got = _run(V, F, P, 40, capture=True)
        for f, t in got:
            samples.add(f, t, 4096, rng)
    feats, targets = samples.arrays()
    assert np.isfinite(feats).all() and np.isfinite(targets).all()
    params, hist = L.train(feats, targets, steps=600, batch=8192, lr=2e-3)
    print(f"{len(feats)} samples, loss {hist[0]:.4f} -> {hist[-1]:.4f}")
    assert hist[-1] < hist[0]

    V, F, P = _pinned_sheet(36, 9)
    plain, taken0, xp, _ = _run(V, F, P, 30)
    learned, taken, xl, _ = _run(V, F, P, 30, params=params, learned=True)
    print(f"first-solve CG iterations: plain {plain}, learned {learned} "
          f"({taken} of 30 learned starts taken)")
    assert taken0 == 0
    assert np.abs(xl - xp).max() < 2e-3

    bad = params.copy()
    for name in ("W4", "b4"):
        L.put(bad, name, np.zeros_like(L.get(bad, name)))
    worse, taken_bad, xb, _ = _run(V, F, P, 30, params=bad, learned=True)
    print(f"zero model: {taken_bad} starts taken, first-solve iterations {worse}")
    assert taken_bad == 0
    assert worse == plain
    np.testing.assert_array_equal(xb, xp)


MODEL = Path(__file__).resolve().parents[1] / "silk_physics_b200" / "models" / "warm_start.npy"
# Held-out gain required of the committed iterate model: CG iterations per
# solve of the learned run at most this fraction of the plain run's.
HELD_OUT_GAIN = 0.97


def _held_out_run(params, learned, extrap=False, steps=2):
    """A scene outside the training mix (seeds, size and radius of its own):
    a 70 x 70 sheet of side 1.2 m over a sphere of radius 0.45 m, from its
    free-fall state one step before contact; default settings, CG relative
    tolerance 1e-5."""
    V, F = S.grid_sheet(70, side=1.2, z=0.55, jitter=1e-4, seed=4242)
    SV, SF = S.icosphere(4, 0.45, center=(0.05, -0.03, 0.0))
    x0, v0 = S.free_fall_state(V, 7)
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5,
                                                learned_warm_start=learned,
                                                admm_extrapolated_start=extrap))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, [])
    assert r
    r, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
    assert r
    if params is not None:
        assert w.set_warm_start_model(params)
    assert w.set_cloth_state(h, x0, v0)
    cg = solves = iter_starts = contacts = 0
    for _ in range(steps):
        r = w.solver_step()
        assert r, r.to_string()
        st = w.step_stats()
        cg += st.cg_iterations
        solves += st.cg_solves
        iter_starts += st.learned_iterate_starts
        contacts = st.contacts
    x = np.zeros(V.size, np.float32)
    assert w.get_cloth_position(h, x)
    return cg / max(solves, 1), iter_starts, contacts, x


@pytest.mark.gpu
def test_trained_model_gains_on_held_out_scene():
    """The committed model file (both networks, trained by
    python -m silk_physics_b200.learned on solver samples of the training mix)
    on a held-out contact scene: the iterate model's starts are taken and the
    CG needs fewer iterations per solve than from the plain start (the
    reference's warm start, the previous ADMM iterate), by at least
    1 - HELD_OUT_GAIN; positions stay within the contact tolerance of the
    plain run.  The ADMM-extrapolated start (2 x_k - x_(k-1)) is printed
    beside them."""
    params = L.load(str(MODEL))
    assert params.size == 2 * L.N_PARAMS
    plain, s0, c0, xp = _held_out_run(None, False)
    learned, s1, c1, xl = _held_out_run(params, True)
    extrap, _, _, _ = _held_out_run(None, False, extrap=True)
    print(f"CG iterations per solve: plain {plain:.2f}, learned {learned:.2f} "
          f"({s1} iterate-model starts), extrapolated {extrap:.2f}; contacts {c0} / {c1}")
    assert s0 == 0 and s1 > 0 and c0 > 0
    assert learned <= HELD_OUT_GAIN * plain
    assert np.abs(xl - xp).max() < 1e-3
