"""State of the 80x80 sheet-on-sphere scene (the benchmark workload) after
its 24 free-fall and 3 warm-up steps, computed by the CPU oracle itself: the
starting point of both arms of bench.py, so that they time the same contact
steps from the same state without replaying 27 steps on the host cores
first.

The file holds x and v (mesh order) after 27 oracle steps (run with banks of
32 consecutive vertices), and perm / part_offsets: the MAS partition both
arms use for the steps after it (the host partition of silk_partition_mesh,
which the CUDA path computes itself), so that the two arms solve with the
same preconditioner.

Run from the repository root:  python oracle/make_reference_state.py
(writes oracle/reference_state_c2_step27.npz; the oracle is deterministic
for any number of OpenMP threads, so the file is reproducible).
"""
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import pyoracle  # noqa: E402

STEPS = 27
OUT = HERE / "reference_state_c2_step27.npz"


def world(cg_rel_tol=1e-5):
    import bench

    V, F, SV, SF = bench.scene()  # noqa: F841
    ow = pyoracle.OracleWorld(config=dict(acceleration=(0.0, 0.0, -9.81),
                                          fixed_linear_rel_tol=cg_rel_tol))
    nv = len(V)
    perm = np.arange(nv, dtype=np.int32)
    offs = np.unique(np.append(np.arange(0, nv, 32), nv)).astype(np.int32)
    h = ow.add_cloth(V, F, [], perm, offs)
    ow.add_obstacle(SV, SF)
    return ow, h, V


def main():
    pyoracle.build()
    ow, h, V = world()
    t = time.perf_counter()
    for k in range(STEPS):
        assert ow.step() == 0
        print(f"step {k + 1}: {time.perf_counter() - t:.1f} s", flush=True)
    from silk_physics_b200 import native as N

    perm, offs = N.partition_mesh(V, bench.scene()[1])
    np.savez_compressed(OUT, x=ow.position_f32(h), v=ow.velocity(h), steps=STEPS, perm=perm,
                        part_offsets=offs)
    print("written", OUT.name)


if __name__ == "__main__":
    main()
