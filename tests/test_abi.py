"""The C-ABI library loads and exports every symbol the header declares."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "silk_b200.h").read_text()
    declared = set(re.findall(r"\b(silk_[a-z0-9_]+)\s*\(", header))
    lib = C.CDLL(str(ROOT / "silk_physics_b200" / "libsilk_b200.so"))
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert len(declared) >= 30


def test_defaults_match_reference_config():
    from silk_physics_b200 import native as N

    c = N._GlobalConfigC()
    N.lib.silk_global_config_default(C.byref(c))
    g = N.GlobalConfig()
    for name, _ in N._GlobalConfigC._fields_:
        assert np.float32(getattr(c, name)) == np.float32(getattr(g, name)), name
    assert c.acceleration_z == -10.0 and c.max_inner_iteration == 100


def test_world_without_init_reports_not_initialized():
    from silk_physics_b200 import native as N

    w = N.World()
    r = w.solver_step()
    assert not r and r.code == N.ErrorCode.NotInitialized
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), [0, 0, 0], [0, 1, 2])
    assert not r and h == 0


def test_cpu_backend_is_not_provided():
    from silk_physics_b200 import native as N

    w = N.World()
    r = w.init(N.Backend.CPU)
    assert not r and r.code == N.ErrorCode.InvalidConfig


def test_partition_rejects_bad_meshes_and_small_buffers():
    """silk_partition_mesh checks sizes, finiteness and face indices before
    partitioning (an index past the vertex count used to read out of
    bounds), and reports the part count when the offsets buffer is short."""
    import pytest

    from silk_physics_b200 import native as N

    V = np.random.default_rng(0).random((10, 3)).astype(np.float32)
    for F in ([[0, 1, 20]], [[0, -1, 2]], [[0, 0, 2]]):
        with pytest.raises(RuntimeError, match="InvalidMesh"):
            N.partition_mesh(V, np.array(F, np.int32))
    bad = V.copy()
    bad[3, 1] = np.nan
    with pytest.raises(RuntimeError, match="InvalidMesh"):
        N.partition_mesh(bad, np.array([[0, 1, 2]], np.int32))
    F = np.array([[0, 1, 2], [1, 2, 3]], np.int32)
    perm = np.zeros(10, np.int32)
    offs = np.zeros(1, np.int32)
    n = C.c_int32(0)
    st = N.lib.silk_partition_mesh(V.ravel(), V.size, F.ravel(), F.size, perm, offs, 1,
                                   C.byref(n))
    assert st == int(N.ErrorCode.InvalidConfig) + 1 and n.value > 0
    perm, offs = N.partition_mesh(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32))
    assert perm.size == 0 and offs.tolist() == [0]


def test_row_schedule_rejects_rows_longer_than_width():
    import pytest

    from silk_physics_b200 import native as N

    rows = [[(-1, 5), (-2, 6)]] + [[] for _ in range(31)]
    with pytest.raises(RuntimeError, match="InvalidConfig"):
        N.schedule_bank_rows(rows, 1, 0)
    cols, vals = N.schedule_bank_rows([[] for _ in range(32)], 0, 0)
    assert cols.shape == (0, 32) and vals.shape == (0, 32)


def test_world_calls_before_init_report_not_initialized():
    from silk_physics_b200 import native as N

    w = N.World()
    x = np.zeros(3, np.float32)
    for r in (w.set_global_config(N.GlobalConfig()), w.remove_cloth(5),
              w.get_cloth_position(1, x), w.set_obstacle_position(1, x),
              w.set_cloth_pin_index(1, [0]), w.solver_reset()):
        assert not r and r.code == N.ErrorCode.NotInitialized
    w.clear()
