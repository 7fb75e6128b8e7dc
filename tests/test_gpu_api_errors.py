"""Error paths of the silk::World API on an initialised GPU world, injected
on the host (the reference's Result codes, silk/include/silk/result.hpp:22-35):
bad pins, wrong spans, unknown and removed handles, and the CG iteration
bound."""
import numpy as np
import pytest

from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

pytestmark = pytest.mark.gpu

NO_COLLISION = N.CollisionConfig(is_collision_on=False, is_self_collision_on=False)


def test_pin_span_and_handle_errors():
    V, F = S.grid_sheet(8)
    w = N.World()
    assert w.init()
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, [0, len(V)])
    assert not r and r.code == N.ErrorCode.InvalidPin and h == 0
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, [0, 7])
    assert r and h != 0
    assert w.set_cloth_pin_index(h, [len(V) + 5]).code == N.ErrorCode.InvalidPin
    assert w.set_cloth_pin_position(h, np.zeros(3, np.float32)).code == N.ErrorCode.InvalidPin
    assert w.set_cloth_pin_position(h, np.zeros(6, np.float32))
    x = np.zeros(V.size - 3, np.float32)
    assert w.get_cloth_position(h, x).code == N.ErrorCode.InvalidPosition
    for bad in (w.remove_cloth(h + 100), w.set_cloth_config(h + 100, N.ClothConfig()),
                w.set_cloth_pin_index(h + 100, [0])):
        assert bad.code == N.ErrorCode.InvalidHandle
    assert w.solver_step()
    assert w.remove_cloth(h)
    assert w.get_cloth_position(h, np.zeros(V.size, np.float32)).code == \
        N.ErrorCode.InvalidHandle


def test_cg_iteration_bound():
    """cg_max_iter bounds every solve; the step still completes, as in the
    reference, which does not act on a CG that stopped at its bound."""
    V, F = S.grid_sheet(24)
    w = N.World()
    assert w.init()
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-9, cg_max_iter=3))
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, S.top_corner_pins(24))
    assert r
    assert w.solver_step()
    st = w.step_stats()
    assert st.cg_solves > 0 and st.cg_iterations <= 3 * st.cg_solves
    x = np.zeros(V.size, np.float32)
    assert w.get_cloth_position(h, x) and np.isfinite(x).all()


def test_gpu_coulomb_known_answers():
    """The GPU contact projection on the reference's known answers
    (test/friction_contact_test.cu:23-63): exact values."""
    n = [0.0, 0.0, 1.0]
    cases = [((1, -2, 0.5), 0.7, [1.0, -2.0, 0.5]),
             ((0.2, 0, -1), 0.5, [0.0, 0.0, 0.0]),
             ((2, 0, -1), 0.5, [1.5, 0.0, 0.0]),
             ((2, -3, -1), 0.0, [2.0, -3.0, 0.0])]
    out = N.debug_coulomb([c[0] for c in cases], [n] * len(cases), [c[1] for c in cases])
    for k, (_, _, want) in enumerate(cases):
        assert out[k].tolist() == want, (k, out[k])


def test_gpu_coulomb_complementarity_and_cone():
    """test/friction_contact_test.cu:65-92 through the GPU projection, with
    the reference's tolerance 1e-5, plus random normals and displacements."""
    us = [(0, 0, 1), (2, -1, 0), (0.1, 0.2, -1), (2, 0, -1), (-3, 4, -0.5), (0, 0, -2)]
    mus = [0.0, 0.1, 0.5, 2.0]
    u = np.array([q for m in mus for q in us], np.float32)
    mu = np.array([m for m in mus for _ in us], np.float32)
    nn = np.tile(np.array([0, 0, 1.0], np.float32), (len(mu), 1))
    rng = np.random.default_rng(5)
    ru = rng.normal(0, 1, (2000, 3)).astype(np.float32)
    rn = rng.normal(0, 1, (2000, 3))
    rn = (rn / np.linalg.norm(rn, axis=1, keepdims=True)).astype(np.float32)
    rmu = rng.uniform(0, 2, 2000).astype(np.float32)
    u, nn, mu = np.concatenate([u, ru]), np.concatenate([nn, rn]), np.concatenate([mu, rmu])
    s = N.debug_coulomb(u, nn, mu).astype(np.float64)
    r = s - u
    sn = np.sum(s * nn, axis=1)
    rnrm = np.sum(r * nn, axis=1)
    rt = r - rnrm[:, None] * nn
    assert np.all(sn >= -1e-5) and np.all(rnrm >= -1e-5)
    assert np.all(np.abs(sn * rnrm) <= 1e-5 * np.maximum(1.0, np.abs(u).max(axis=1)) ** 2)
    assert np.all(np.linalg.norm(rt, axis=1) <= mu * rnrm + 1e-5 * np.maximum(
        1.0, np.abs(u).max(axis=1)))


def test_gpu_coulomb_matches_oracle(oracle):
    """The GPU projection's one-rsqrt form against the oracle's restatement of
    the reference's sqrt-and-divide form: a few ulp apart at most."""
    import ctypes as C

    rng = np.random.default_rng(11)
    n = 4000
    u = rng.normal(0, 1, (n, 3)).astype(np.float32)
    nn = rng.normal(0, 1, (n, 3))
    nn = (nn / np.linalg.norm(nn, axis=1, keepdims=True)).astype(np.float32)
    mu = rng.uniform(0, 1.5, n).astype(np.float32)
    g = N.debug_coulomb(u, nn, mu)
    L = oracle.lib()
    f3 = C.c_float * 3
    for i in range(n):
        out = f3()
        L.oracle_solve_coulomb(f3(*u[i]), f3(*nn[i]), C.c_float(mu[i]), out)
        o = np.array(list(out), np.float32)
        np.testing.assert_allclose(g[i], o, rtol=4e-6, atol=4e-7 * float(np.abs(u[i]).max()),
                                   err_msg=str(i))


def test_mas_pivot_failure_reported():
    """A non-finite bank matrix (density NaN makes the mass diagonal NaN) is
    caught by the bank inversion's pivot check and reported as
    IterativeSolveFail, as the reference rejects a failed packed inverse
    (mas_preconditioner.cu:854-858).  The world stays usable."""
    V, F = S.grid_sheet(12)
    w = N.World()
    assert w.init()
    r, h = w.add_cloth(N.ClothConfig(density=float("nan")), NO_COLLISION, V, F, [])
    assert r
    r = w.solver_step()
    assert r.code == N.ErrorCode.IterativeSolveFail, r.to_string()
    assert "MAS bank inverse" in r.detail, r.detail
    assert w.set_cloth_config(h, N.ClothConfig())
    assert w.set_cloth_state(h, V)
    r = w.solver_step()
    assert r, r.to_string()


def test_grid_barrier_wait_runs_out():
    """A cooperative-grid CG launch in which one block never arrives at its
    barriers (test switch debug_withhold_block): the other blocks' waits end
    after barrier_spin_limit polls, the kernel returns, the step reports
    IterativeSolveFail, and the same world steps normally afterwards."""
    V, F = S.grid_sheet(160, side=1.0, z=1.0)
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(max_inner_iteration=4))
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, [])
    assert r
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5,
                                                barrier_spin_limit=1 << 16,
                                                debug_withhold_block=1))
    r = w.solver_step()
    assert r.code == N.ErrorCode.IterativeSolveFail, r.to_string()
    assert "barrier" in r.detail, r.detail
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5))
    assert w.set_cloth_state(h, V)
    r = w.solver_step()
    assert r, r.to_string()
    assert w.step_stats().cg_resident_solves > 0


def test_set_state_continues_the_same_trajectory():
    """Positions and velocities are the whole state between steps: a world
    restarted from another world's (x, v) takes the identical next step."""
    V, F = S.grid_sheet(24, side=0.5, z=0.35, jitter=1e-4, seed=2)
    SV, SF = S.icosphere(2, radius=0.3)

    def world():
        w = N.World()
        assert w.init()
        assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81))
        assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5))
        r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, [])
        assert r
        r, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
        assert r
        return w, h

    a, ha = world()
    for _ in range(4):
        assert a.solver_step()
    x = np.zeros(V.size, np.float32)
    v = np.zeros(V.size, np.float32)
    assert a.get_cloth_position(ha, x)
    assert a.get_cloth_velocity(ha, v)
    b, hb = world()
    assert b.set_cloth_state(hb, x, v)
    xb = np.zeros_like(x)
    assert b.get_cloth_position(hb, xb)
    np.testing.assert_array_equal(xb, x)
    for _ in range(2):
        assert a.solver_step()
        assert b.solver_step()
        sa, sb = a.step_stats(), b.step_stats()
        assert (sa.contacts, sa.admm_iterations, sa.cg_iterations) == \
            (sb.contacts, sb.admm_iterations, sb.cg_iterations)
    xa = np.zeros_like(x)
    assert a.get_cloth_position(ha, xa)
    assert b.get_cloth_position(hb, xb)
    np.testing.assert_array_equal(xa, xb)
    bad = x.copy()
    bad[5] = np.nan
    assert b.set_cloth_state(hb, bad).code == N.ErrorCode.InvalidPosition
