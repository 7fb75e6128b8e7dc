"""GPU solver path against the oracle: ADMM + MAS-PCG + pins (no contacts)."""
import numpy as np
import pytest

from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

pytestmark = pytest.mark.gpu

NO_COLLISION = N.CollisionConfig(is_collision_on=False, is_self_collision_on=False)


def _pair(oracle, s, steps, fp64=False, inner=10, admm_tol=0.0, cg_rel=1e-6, bf16=False,
          pins=True, cloth=None, jitter=0.0):
    V, F = S.grid_sheet(s, jitter=jitter, seed=7)
    P = S.top_corner_pins(s) if pins else np.zeros(0, np.int32)
    cloth = cloth or N.ClothConfig()
    g = N.GlobalConfig(max_inner_iteration=inner, admm_abs_tol=admm_tol, admm_rel_tol=admm_tol)
    w = N.World()
    assert w.init()
    assert w.set_global_config(g)
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=cg_rel, mas_bf16=bf16))
    r, h = w.add_cloth(cloth, NO_COLLISION, V, F, P)
    assert r, r.to_string()
    perm, offs = w.cloth_partition(h, len(V))
    ow = oracle.OracleWorld(fp64=fp64, config=dict(
        max_inner_iteration=inner, admm_abs_tol=admm_tol, admm_rel_tol=admm_tol,
        fixed_linear_rel_tol=cg_rel))
    oh = ow.add_cloth(V, F, P, perm, offs,
                      cloth=(cloth.elastic_stiffness, cloth.bending_stiffness,
                             cloth.density, cloth.damping),
                      collision=(0, 0, 0, 0.3, 0.3))
    out = []
    x = np.zeros(3 * len(V), np.float32)
    for k in range(steps):
        assert w.solver_step()
        assert ow.step() == 0
        assert w.get_cloth_position(h, x)
        out.append((k + 1, x.reshape(-1, 3).astype(np.float64).copy(), ow.position(oh)))
    return w, h, ow, out, V


def test_position_before_step_is_rest_state():
    V, F = S.grid_sheet(8)
    w = N.World()
    assert w.init()
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, [])
    assert r and h != 0
    x = np.zeros(V.size, np.float32)
    assert w.get_cloth_position(h, x)
    np.testing.assert_array_equal(x.reshape(-1, 3), V)
    bad = np.zeros(V.size - 3, np.float32)
    r = w.get_cloth_position(h, bad)
    assert not r and r.code == N.ErrorCode.InvalidPosition
    r = w.get_cloth_position(h + 100, x)
    assert not r and r.code == N.ErrorCode.InvalidHandle


@pytest.mark.parametrize("steps", [1, 10])
def test_sheet32_matches_fp32_oracle(oracle, steps):
    """Config 1 shape (32x32 sheet, two top corners pinned, 10 ADMM
    iterations): positions after 1 and 10 steps within 2e-5 m of the FP32
    oracle running the same algorithm."""
    _, _, _, out, _ = _pair(oracle, 32, steps)
    for k, xg, xo in out:
        err = np.abs(xg - xo).max()
        print(f"step {k}: max |gpu - oracle32| = {err:.3e}")
        assert err < 2e-5, (k, err)


def test_sheet32_error_vs_fp64_oracle(oracle):
    _, _, _, out, _ = _pair(oracle, 32, 10, fp64=True, cg_rel=1e-6)
    k, xg, xo = out[-1]
    err = np.abs(xg - xo).max()
    print(f"10 steps: max |gpu - oracle64| = {err:.3e}")
    assert err < 5e-5


def test_pins_hold_and_sheet_falls(oracle):
    w, h, _, out, V = _pair(oracle, 24, 10)
    x = out[-1][1]
    P = S.top_corner_pins(24)
    np.testing.assert_allclose(x[P], V[P], atol=1e-6)
    assert x[:, 2].min() < V[:, 2].min() - 0.01
    st = w.step_stats()
    assert st.cg_iterations > 0 and st.admm_iterations == 10 and st.kernel_launches > 0


def test_default_tolerances_match_oracle(oracle):
    """Reference adaptive CG tolerance and ADMM stopping rule."""
    _, _, _, out, _ = _pair(oracle, 20, 5, inner=100, admm_tol=None or 1e-5, cg_rel=0.0,
                            jitter=1e-4)
    for k, xg, xo in out:
        err = np.abs(xg - xo).max()
        print(f"step {k}: default tolerances max err {err:.3e}")
        assert err < 2e-4


def test_bf16_mas_converges_to_same_solution(oracle):
    _, _, _, out32, _ = _pair(oracle, 32, 3, cg_rel=1e-6)
    _, _, _, outbf, _ = _pair(oracle, 32, 3, cg_rel=1e-6, bf16=True)
    err = np.abs(out32[-1][1] - outbf[-1][1]).max()
    print(f"bf16 vs fp32 MAS after 3 steps: {err:.3e}")
    assert err < 2e-5


def test_solver_reset_restores_rest_state():
    V, F = S.grid_sheet(10)
    w = N.World()
    assert w.init()
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, [])
    assert w.solver_step()
    x = np.zeros(V.size, np.float32)
    assert w.get_cloth_position(h, x)
    assert np.abs(x.reshape(-1, 3) - V).max() > 0
    assert w.solver_reset()
    assert w.get_cloth_position(h, x)
    np.testing.assert_array_equal(x.reshape(-1, 3), V)
    assert w.remove_cloth(h)
    r = w.solver_step()
    assert not r and r.code == N.ErrorCode.Unknown
