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
