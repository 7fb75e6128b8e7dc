"""B200-native per-step cloth simulation (the silk::World hot path).

The native library ``libsilk_b200.so`` (CUDA kernels for sm_100a behind the C
ABI of ``include/silk_b200.h``) does all the work; ``silk_physics_b200.native``
is a thin Python mirror of ``silk::World`` (silk/include/silk/silk.hpp:83-239)
with the same method names, argument meaning and ``Result`` / ``ErrorCode``
values (silk/include/silk/result.hpp:22-80).  There is no CPU fallback: using
the package fails loudly when the library is missing.

The native module is loaded on first attribute access so that
``python -m silk_physics_b200.build`` can run before the library exists.
"""
from __future__ import annotations

_EXPORTS = {
    "Backend", "ClothConfig", "CollisionConfig", "ErrorCode", "GlobalConfig", "Result",
    "SolverOptions", "StepStats", "World", "ccd_batch", "color_contacts", "lib",
    "partition_mesh", "assemble_cloth_host",
}


def __getattr__(name: str):
    if name in _EXPORTS:
        from . import native

        return getattr(native, name)
    raise AttributeError(name)
