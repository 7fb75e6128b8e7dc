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
