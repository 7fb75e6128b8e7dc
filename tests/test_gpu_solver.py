"""GPU solver path against the oracle: ADMM + MAS-PCG + pins (no contacts)."""
from pathlib import Path

import numpy as np
import pytest

from silk_physics_b200 import native as N
from silk_physics_b200 import scenes as S

pytestmark = pytest.mark.gpu

NO_COLLISION = N.CollisionConfig(is_collision_on=False, is_self_collision_on=False)


def _pair(oracle, s, steps, fp64=False, inner=10, admm_tol=0.0, cg_rel=1e-6, bf16=False,
          pins=True, cloth=None, jitter=0.0, form=0, extrap=False, halo_limit=0):
    V, F = S.grid_sheet(s, jitter=jitter, seed=7)
    P = S.top_corner_pins(s) if pins else np.zeros(0, np.int32)
    cloth = cloth or N.ClothConfig()
    g = N.GlobalConfig(max_inner_iteration=inner, admm_abs_tol=admm_tol, admm_rel_tol=admm_tol)
    w = N.World()
    assert w.init()
    assert w.set_global_config(g)
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=cg_rel, mas_bf16=bf16,
                                                cg_form=form, admm_extrapolated_start=extrap,
                                                resident_halo_limit=halo_limit))
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


def test_sheet32_parity_with_oracle(oracle):
    """Config 1 shape (32x32 sheet, two top corners pinned, 10 ADMM
    iterations, CG rel 1e-6).  Ten un-converged ADMM iterations amplify FP32
    rounding, so the FP32 restatement itself drifts from the FP64 solution
    (about 1e-5 m after one step, 4e-4 m after ten).  The GPU must stay within
    the stated tolerance of the FP32 oracle (1e-4 m after 1 step, 2e-3 m after
    10) and be no further from the FP64 solution than three times the FP32
    oracle's own drift (floor 2e-5 m)."""
    _, _, _, o32, _ = _pair(oracle, 32, 10)
    _, _, _, o64, _ = _pair(oracle, 32, 10, fp64=True)
    for (k, xg, x32), (_, _, x64) in zip(o32, o64):
        e32 = np.abs(xg - x32).max()
        eg64 = np.abs(xg - x64).max()
        e3264 = np.abs(x32 - x64).max()
        print(f"step {k}: |gpu-o32| {e32:.2e} |gpu-o64| {eg64:.2e} |o32-o64| {e3264:.2e}")
        if k == 1:
            assert e32 < 1e-4
        if k == 10:
            assert e32 < 2e-3
        assert eg64 <= max(3.0 * e3264, 2e-5)


def test_well_conditioned_parity(oracle):
    """Heavier, softer cloth and converged ADMM: the FP32 noise floor is low
    (FP32 vs FP64 oracle: 6e-7 m after 1 step, 7e-6 m after 10), so GPU and
    FP32 oracle agree to 5e-6 m after 1 step and 5e-5 m after 10."""
    cloth = N.ClothConfig(elastic_stiffness=10.0, bending_stiffness=1e-4, density=5.0,
                          damping=0.01)
    _, _, _, out, _ = _pair(oracle, 24, 10, inner=50, admm_tol=1e-6, cg_rel=1e-6,
                            cloth=cloth)
    for k, xg, xo in out:
        err = np.abs(xg - xo).max()
        print(f"step {k}: well-conditioned |gpu-o32| = {err:.3e}")
        if k == 1:
            assert err < 5e-6
        if k == 10:
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
    _, _, _, out, _ = _pair(oracle, 20, 5, inner=100, admm_tol=1e-5, cg_rel=0.0,
                            jitter=1e-4)
    for k, xg, xo in out:
        err = np.abs(xg - xo).max()
        print(f"step {k}: default tolerances max err {err:.3e}")
        assert err < 5e-4


def test_bf16_mas_converges_to_same_solution(oracle):
    _, _, _, out32, _ = _pair(oracle, 32, 3, cg_rel=1e-6)
    _, _, _, outbf, _ = _pair(oracle, 32, 3, cg_rel=1e-6, bf16=True)
    err = np.abs(out32[-1][1] - outbf[-1][1]).max()
    print(f"bf16 vs fp32 MAS after 3 steps: {err:.3e}")
    assert err < 2e-4


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


def _gpu_run(s, steps, form, tol=1e-5, jitter=1e-4):
    V, F = S.grid_sheet(s, jitter=jitter, seed=3)
    P = S.top_corner_pins(s)
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(max_inner_iteration=10, admm_abs_tol=0.0,
                                              admm_rel_tol=0.0))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=tol, cg_form=form))
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, P)
    assert r
    iters, resident = [], 0
    for _ in range(steps):
        assert w.solver_step(), w
        st = w.step_stats()
        iters.append(st.cg_iterations)
        resident += st.cg_resident_solves
    return iters, resident


# Form 0 (default): 32 -> the cluster form with redundant coarse levels on 5
# CTAs of 8 fine banks; 80 -> the same on 14 CTAs of 16; 128 -> too many fine
# banks for one such cluster: the resident form, a cooperative grid of 17
# blocks.  Form 2 (resident): 32 a 2-block cluster, 80 a 7-block cluster,
# 128 the grid.  Form 1: streaming.
@pytest.mark.parametrize("s", [32, 80, 128])
def test_resident_and_streaming_forms_against_oracle(oracle, s):
    """The cluster form with redundant coarse levels, the resident CG kernel
    (one block per first-level coarse bank) and the streaming kernel run the
    same preconditioned iteration and differ only in the order of FP64 sums,
    of the off-diagonal terms of a row and of the coarse bank solves.  In the
    well-conditioned, converged setting each form must be as close to the
    FP64 oracle as 3x the FP32 oracle's own drift (floor 2e-6 m; the drift
    grows with the mesh: about 1e-6 m at 32x32, 6e-6 m at 128x128); in the
    default setting their CG iteration counts agree within 5 %."""
    cloth = N.ClothConfig(elastic_stiffness=10.0, bending_stiffness=1e-4, density=5.0,
                          damping=0.01)
    kw = dict(inner=50, admm_tol=1e-6, cg_rel=1e-6, cloth=cloth, jitter=1e-4)
    _, _, _, o32, _ = _pair(oracle, s, 1, **kw)
    _, _, _, o64, _ = _pair(oracle, s, 1, fp64=True, **kw)
    e3264 = np.abs(o32[0][2] - o64[0][2]).max()
    for form in (0, 2, 1):
        w, _, _, og, _ = _pair(oracle, s, 1, form=form, **kw)
        st = w.step_stats()
        eg64 = np.abs(og[0][1] - o64[0][2]).max()
        print(f"s={s} form={form}: |gpu-o64| {eg64:.2e} |o32-o64| {e3264:.2e}, "
              f"cluster solves {st.cg_cluster_solves} resident {st.cg_resident_solves} "
              f"of {st.cg_solves}")
        assert eg64 <= max(3.0 * e3264, 2e-6)
        if form == 0:
            assert (st.cg_cluster_solves == st.cg_solves) == (s <= 80)
        else:
            assert st.cg_cluster_solves == 0
    ic, ncl = _gpu_run(s, 3, 0)
    ir, nres = _gpu_run(s, 3, 2)
    is_, nstr = _gpu_run(s, 3, 1)
    print(f"s={s}: CG iterations default {ic} resident {ir} streaming {is_}")
    assert nres > 0 and nstr == 0
    assert all(abs(a - b) <= 0.05 * b for a, b in zip(ir, is_))
    assert all(abs(a - b) <= 0.05 * b for a, b in zip(ic, is_))


# (cg_form with rows in tensor memory, the same with rows in global memory,
# sheet side): the cluster form on 5 CTAs of 8 fine banks and on 14 of 16;
# the resident form as a 2- and a 7-block cluster and a 17-block cooperative
# grid.
ROW_STORE_CASES = [(0, 3, 32), (0, 3, 80), (2, 4, 32), (2, 4, 80), (2, 4, 128)]


@pytest.mark.parametrize("form_tm,form_global,s", ROW_STORE_CASES)
@pytest.mark.parametrize("bf16", [False, True])
def test_cg_rows_tensor_memory_identical(form_tm, form_global, s, bf16):
    """The cluster and resident CG forms hold their SpMV rows in tensor
    memory (cg_form 0 and 2) or read them from global memory in every SpMV
    (cg_form 3 and 4): the same entries in the same order, so bit-identical
    positions and iteration counts after three steps."""
    out = []
    for form in (form_tm, form_global):
        V, F = S.grid_sheet(s, jitter=1e-4, seed=3)
        w = N.World()
        assert w.init()
        assert w.set_global_config(N.GlobalConfig(max_inner_iteration=10))
        assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5, cg_form=form,
                                                    mas_bf16=bf16))
        r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, S.top_corner_pins(s))
        assert r
        iters = []
        for _ in range(3):
            assert w.solver_step(), w
            st = w.step_stats()
            if form_tm == 0:
                assert st.cg_cluster_solves == st.cg_solves > 0
            else:
                assert st.cg_resident_solves == st.cg_solves > 0 and st.cg_cluster_solves == 0
            iters.append(st.cg_iterations)
        x = np.zeros(V.size, np.float32)
        assert w.get_cloth_position(h, x)
        out.append((iters, x))
    print(f"forms {form_tm}/{form_global} s={s} bf16={bf16}: CG iterations {out[0][0]} "
          f"(tensor memory) {out[1][0]} (global)")
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("interval", [2, 4, 7])
def test_device_decided_admm_iterations_identical(interval):
    """The host reads the device's ADMM convergence state every
    admm_check_interval iterations (1: after each, the reference's loop);
    the iterations enqueued after convergence find AdmmControl::done set and
    do nothing.  On the 80x80 contact scene from the stored state (three
    steps: ADMM solves of tens to hundreds of iterations, CCD rollbacks,
    contacts) and on config 1 (10 iterations, never converged): bit-identical
    positions and the same ADMM / CG / contact counts."""
    from silk_physics_b200 import scenes as SC
    g = np.load(Path(__file__).resolve().parent / "golden" / "c2_contact.npz")
    V, F, SV, SF = SC.c2_scene()

    def run(iv, scene):
        w = N.World()
        assert w.init()
        if scene == "c2":
            assert w.set_global_config(N.GlobalConfig(acceleration_z=-9.81))
            assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5,
                                                        admm_check_interval=iv))
            r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, [])
            assert r
            r, _ = w.add_obstacle(N.CollisionConfig(), SV, SF)
            assert r
            assert w.set_cloth_state(h, g["x0"], g["v0"])
            n, steps = len(V), 3
        else:
            V1, F1 = S.grid_sheet(32, jitter=0.0, seed=7)
            assert w.set_global_config(N.GlobalConfig(max_inner_iteration=10, admm_abs_tol=0.0,
                                                      admm_rel_tol=0.0))
            assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-5,
                                                        admm_check_interval=iv))
            r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V1, F1,
                               S.top_corner_pins(32))
            assert r
            n, steps = len(V1), 4
        counts = []
        for _ in range(steps):
            assert w.solver_step(), w
            st = w.step_stats()
            counts.append((st.admm_iterations, st.cg_iterations, st.cg_solves, st.contacts,
                           st.outer_iterations, st.cg_resident_solves, st.cg_cluster_solves))
        x = np.zeros(3 * n, np.float32)
        assert w.get_cloth_position(h, x)
        return counts, x

    for scene in ("c2", "c1"):
        c_ref, x_ref = run(1, scene)
        c, x = run(interval, scene)
        print(f"{scene} interval {interval}: (ADMM, CG, solves, contacts, outer, resident, cluster) "
              f"{c} vs every iteration {c_ref}")
        assert c == c_ref
        np.testing.assert_array_equal(x, x_ref)


@pytest.mark.parametrize("form", [0, 1])
def test_admm_extrapolated_start_against_oracle(oracle, form):
    """CG solves started from 2 x_k - x_(k-1) of the ADMM iterates (blended
    with the plain start by the residual-minimising weight, stopping rule
    judged by the plain start's residual) reach the same ADMM result.  Config
    1 setting (default cloth, 30 un-converged ADMM iterations, CG rel 1e-6)
    on a 48x48 sheet: within the FP32 parity bound of the FP64 oracle (or of
    the plain start's own distance to it) after 3 steps in both CG forms, the
    extrapolated start taken in most solves and
    no more CG iterations than from the plain start (5 % allowance)."""
    kw = dict(inner=30, cg_rel=1e-6, jitter=1e-4, form=form)
    _, _, _, o32, _ = _pair(oracle, 48, 3, **kw)
    _, _, _, o64, _ = _pair(oracle, 48, 3, fp64=True, **kw)
    wp, _, _, op, _ = _pair(oracle, 48, 3, **kw)
    we, _, _, oe, _ = _pair(oracle, 48, 3, extrap=True, **kw)
    sp, se = wp.step_stats(), we.step_stats()
    e3264 = np.abs(o32[-1][2] - o64[-1][2]).max()
    ep64 = np.abs(op[-1][1] - o64[-1][2]).max()
    eg64 = np.abs(oe[-1][1] - o64[-1][2]).max()
    print(f"form={form}: |extrapolated-o64| {eg64:.2e} |plain-o64| {ep64:.2e} "
          f"|o32-o64| {e3264:.2e}; CG iterations {sp.cg_iterations} plain, "
          f"{se.cg_iterations} extrapolated ({se.extrapolated_starts} of {se.cg_solves} solves)")
    # Another start gives another (equally converged) CG result, and 30
    # un-converged ADMM iterations amplify such differences like FP32 noise:
    # the extrapolated run must be as close to the FP64 oracle as 3x the FP32
    # oracle's drift, or no further than 1.25x the plain-start GPU run.
    assert eg64 <= max(3.0 * e3264, 1.25 * ep64, 2e-5)
    assert sp.extrapolated_starts == 0
    assert se.extrapolated_starts > se.cg_solves // 2
    # Without contact the ADMM iterates change little between solves and the
    # gain is within noise; the contact benchmark measures it.
    assert se.cg_iterations <= 1.05 * sp.cg_iterations


def test_two_cloths_concurrent_cg_against_oracle(oracle):
    """Two pinned sheets of different sizes in one world: their CG solves run
    concurrently on per-cloth streams (each a thread-block cluster); both
    stay within the FP32 parity bound of the FP64 oracle after two steps."""
    sheets = [(24, 11, 0.0), (32, 12, 2.0)]
    g = dict(max_inner_iteration=10, admm_abs_tol=0.0, admm_rel_tol=0.0,
             fixed_linear_rel_tol=1e-6)
    w = N.World()
    assert w.init()
    assert w.set_global_config(N.GlobalConfig(max_inner_iteration=10, admm_abs_tol=0.0,
                                              admm_rel_tol=0.0))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-6))
    o32 = oracle.OracleWorld(config=g)
    o64 = oracle.OracleWorld(fp64=True, config=g)
    hs = []
    for s, seed, x0 in sheets:
        V, F = S.grid_sheet(s, jitter=1e-4, seed=seed, center=(x0, 0.0))
        P = S.top_corner_pins(s)
        r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, P)
        assert r
        perm, offs = w.cloth_partition(h, len(V))
        h32 = o32.add_cloth(V, F, P, perm, offs, collision=(0, 0, 0, 0.3, 0.3))
        h64 = o64.add_cloth(V, F, P, perm, offs, collision=(0, 0, 0, 0.3, 0.3))
        hs.append((h, h32, h64, V))
    for _ in range(2):
        assert w.solver_step(), w
        assert o32.step() == 0 and o64.step() == 0
    for h, h32, h64, V in hs:
        x = np.zeros(V.size, np.float32)
        assert w.get_cloth_position(h, x)
        xg = x.reshape(-1, 3).astype(np.float64)
        e3264 = np.abs(o32.position(h32) - o64.position(h64)).max()
        eg64 = np.abs(xg - o64.position(h64)).max()
        print(f"cloth {h}: |gpu-o64| {eg64:.2e} |o32-o64| {e3264:.2e}")
        assert eg64 <= max(3.0 * e3264, 2e-5)



@pytest.mark.parametrize("s", [80, 128])
def test_resident_halo_overflow_against_oracle(oracle, s):
    """Halo limit 16 (solver option): every block of the resident CG reads
    more vertices outside itself than its halo holds, so p is published
    through the cluster or grid and the overflow columns are read from
    global memory.  Same parity bound as the full-halo form: within 3x the
    FP32 oracle's drift of the FP64 oracle (floor 2e-6 m), resident form in
    use (cg_form 2; 80: a 7-block cluster; 128: a 17-block cooperative
    grid)."""
    cloth = N.ClothConfig(elastic_stiffness=10.0, bending_stiffness=1e-4, density=5.0,
                          damping=0.01)
    kw = dict(inner=50, admm_tol=1e-6, cg_rel=1e-6, cloth=cloth, jitter=1e-4)
    _, _, _, o32, _ = _pair(oracle, s, 1, **kw)
    _, _, _, o64, _ = _pair(oracle, s, 1, fp64=True, **kw)
    e3264 = np.abs(o32[0][2] - o64[0][2]).max()
    w, _, _, og, _ = _pair(oracle, s, 1, halo_limit=16, form=2, **kw)
    st = w.step_stats()
    eg64 = np.abs(og[0][1] - o64[0][2]).max()
    print(f"s={s} halo limit 16: |gpu-o64| {eg64:.2e} |o32-o64| {e3264:.2e}, "
          f"resident solves {st.cg_resident_solves} of {st.cg_solves}")
    assert st.cg_resident_solves == st.cg_solves > 0
    assert eg64 <= max(3.0 * e3264, 2e-6)


def test_mas_fine_inverses():
    """MAS factorisation (mas_preconditioner.cu:903-965): every fine bank's
    FP32 inverse (built and inverted in FP64) times the bank matrix, L + the
    ADMM diagonal restricted to the bank, is the identity to FP32 rounding
    (max |A A^-1 - I| < 1e-5; measured 2.3e-7); pinned vertices' banks
    included."""
    s = 32
    V, F = S.grid_sheet(s, jitter=1e-4, seed=7)
    P = S.top_corner_pins(s)
    w = N.World()
    assert w.init()
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=1e-6))
    r, h = w.add_cloth(N.ClothConfig(), NO_COLLISION, V, F, P)
    assert r
    assert w.solver_step()
    perm, offs = w.cloth_partition(h, len(V))
    L = w.cloth_matrix(h, len(V))
    inv, diag = w.mas_fine(h, len(offs) - 1, len(V))
    iu = np.triu_indices(32)
    worst = 0.0
    for b in range(len(offs) - 1):
        idx = np.arange(offs[b], offs[b + 1])
        n = len(idx)
        full = np.zeros((32, 32))
        # Packed upper triangle, row by row (i <= j).
        full[iu] = inv[b]
        full = full + np.triu(full, 1).T
        A = L[np.ix_(idx, idx)] + np.diag(diag[idx].astype(np.float64))
        E = A @ full[:n, :n] - np.eye(n)
        worst = max(worst, float(np.abs(E).max()))
    print(f"{len(offs) - 1} banks, max |A A^-1 - I| = {worst:.2e}")
    assert worst < 1e-5
