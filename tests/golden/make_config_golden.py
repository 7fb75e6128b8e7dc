"""Generate the per-configuration parity fixtures of this directory from the
CPU oracle (the restatement of the reference algorithm in oracle/), in FP32
and FP64 solver arithmetic:

* c2_rest.npz: the 6.4K-vertex sheet on the sphere (silk_physics_b200.scenes
  .c2_scene), positions after steps 1 and 10 from rest;
* c2_contact.npz: the same scene restarted from the oracle's stored state
  after 27 steps (oracle/reference_state_c2_step27.npz, in contact), the
  positions after one more step and its contact, colour and outer-iteration
  counts;
* c3_rest.npz: the 100K-vertex drape (scenes.c3_scene), positions after one
  step from rest;
* c3_contact.npz: the drape restarted from its free-fall state after 8 steps
  (scenes.free_fall_state: 3.7 mm above the sphere, falling at 1.26 m/s),
  positions after the first contact step and its counts, with at most 10
  ADMM iterations per outer iteration (as config 1): that step takes over
  twenty CCD rollbacks, and with the default 100 the oracle needs hours per
  precision on the host cores.  The start state is recomputed by
  scenes.free_fall_state (its checksum is stored).

Every case runs the benchmark settings: gravity -9.81, default cloth,
collision and ADMM configuration, CG relative tolerance fixed at 1e-5, the
MAS partition of the host setup (silk_partition_mesh, no GPU needed).
Positions are stored as float32.  The C2 cases take minutes, the C3 cases
much longer, on all host cores.

Run from the repository root:
  python tests/golden/make_config_golden.py c2_rest c2_contact c3_rest c3_contact
"""
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import pyoracle  # noqa: E402
from silk_physics_b200 import native as N  # noqa: E402
from silk_physics_b200 import scenes as S  # noqa: E402

CONFIG = dict(acceleration=(0.0, 0.0, -9.81), fixed_linear_rel_tol=1e-5)
# Per-case changes of the global configuration.
CASE_CONFIG = {"c3_contact": dict(max_inner_iteration=10)}
STAT_KEYS = ("outer_iterations", "admm_iterations", "cg_iterations", "cg_solves", "contacts",
             "colors", "ccd_queries", "ccd_hits", "min_toi")


def scene(name):
    if name.startswith("c2"):
        return S.c2_scene()
    return S.c3_scene()


def start_state(name, V):
    if name == "c2_contact":
        st = np.load(ROOT / "oracle" / "reference_state_c2_step27.npz")
        return st["x"].reshape(-1, 3), st["v"].reshape(-1, 3), int(st["steps"])
    if name == "c3_contact":
        x, v = S.free_fall_state(V, 8)
        return x, v, 8
    return None, None, 0


def steps_of(name):
    return (1, 10) if name == "c2_rest" else (1,)


def run(name):
    V, F, SV, SF = scene(name)
    perm, offs = N.partition_mesh(V, F)
    x0, v0, start = start_state(name, V)
    out = {"perm": perm, "part_offsets": offs, "start_step": np.int32(start),
           "verts_checksum": np.float64(np.asarray(V, np.float64).sum())}
    if x0 is not None and name == "c3_contact":
        out["x0_checksum"] = np.float64(np.asarray(x0, np.float64).sum())
        out["v0_checksum"] = np.float64(np.asarray(v0, np.float64).sum())
    elif x0 is not None:
        out["x0"] = x0.astype(np.float32)
        out["v0"] = v0.astype(np.float32)
    cfg = dict(CONFIG, **CASE_CONFIG.get(name, {}))
    out["max_inner_iteration"] = np.int32(cfg.get("max_inner_iteration", 100))
    for tag, fp64 in (("o32", False), ("o64", True)):
        ow = pyoracle.OracleWorld(fp64=fp64, config=cfg)
        h = ow.add_cloth(V, F, [], perm, offs)
        ow.add_obstacle(SV, SF)
        if x0 is not None:
            ow.set_state(h, x0, v0)
        t0 = time.perf_counter()
        for k in range(1, max(steps_of(name)) + 1):
            assert ow.step() == 0
            st = ow.stats()
            print(f"{name} {tag} step {k}: {st} ({time.perf_counter() - t0:.0f} s)", flush=True)
            if k in steps_of(name):
                out[f"{tag}_step{k}"] = ow.position(h).astype(np.float32)
                for key in STAT_KEYS:
                    out[f"{tag}_step{k}_{key}"] = np.float64(st[key])
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print("written", HERE / f"{name}.npz", flush=True)


def main(names):
    pyoracle.build()
    for n in names:
        run(n)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c2_rest", "c2_contact"])
