"""Batched step of independent worlds (silk_step_many): each world on its
own stream, driven by a pool of host threads; the results equal those of
stepping the same worlds one after another, bit for bit (every reduction and
ordering of the step is deterministic)."""
import numpy as np
import pytest

from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _scene(side, radius, seed):
    V, F = S.grid_sheet(side, side=0.8, z=radius + 0.03, jitter=1e-4, seed=seed)
    SV, SF = S.icosphere(3, radius=radius, center=(0.05 * seed, -0.03 * seed, 0.0))
    return V, F, SV, SF


def _world(V, F, SV, SF):
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81, max_inner_iteration=30))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, [])
    r2, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
    assert r and r2
    return w, h


def test_step_many_equals_sequential_steps():
    scenes = [_scene(24, 0.25, 1), _scene(40, 0.3, 2), _scene(32, 0.2, 3), _scene(48, 0.35, 4)]
    batch = [_world(*sc) for sc in scenes]
    seq = [_world(*sc) for sc in scenes]
    contacts = 0
    for _ in range(6):
        res = N.step_many([w for w, _ in batch], threads=4)
        assert all(res), [r.to_string() for r in res]
        for w, _ in seq:
            assert w.solver_step(), w
        contacts += sum(w.step_stats().contacts for w, _ in seq)
    for (wb, hb), (ws, hs), (V, _, _, _) in zip(batch, seq, scenes):
        xb = np.zeros(V.size, np.float32)
        xs = np.zeros(V.size, np.float32)
        assert wb.get_cloth_position(hb, xb) and ws.get_cloth_position(hs, xs)
        np.testing.assert_array_equal(xb, xs)
    print(f"contacts summed over steps and scenes: {contacts}")
    assert contacts > 0


def test_step_many_rejects_repeated_or_missing_worlds():
    import ctypes as C

    w, _ = _world(*_scene(16, 0.2, 5))
    invalid = int(N.ErrorCode.InvalidConfig) + 1
    arr = (C.c_void_p * 2)(w._w, w._w)
    st = (C.c_int * 2)()
    assert N.lib.silk_step_many(arr, 2, 0, st) == invalid
    assert N.lib.silk_step_many(None, 1, 0, st) == invalid
    assert N.lib.silk_step_many(arr, 0, 0, st) == 0
