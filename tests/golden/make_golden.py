"""Generate the golden fixtures of this directory from the CPU oracle (the
restatement of the reference algorithm in oracle/), on seeded inputs:

* c1_sheet32.npz: the 32x32 sheet with its two top corners pinned, 10 ADMM
  iterations per step, CG relative tolerance 1e-6 (the C1 parity setting),
  collision off, with the MAS partition (host setup, no GPU), and the FP64
  and FP32 oracle positions after steps 1, 5 and 10;
* c1_sheet32_selfcol.npz: the same with the default collision settings
  (collision and self-collision on, as config 1 states), plus the oracle's
  contact counts after those steps;
* ccd_queries.npz: 256 vertex-face and 256 edge-edge Tight-Inclusion CCD
  queries (seeded motions, min separations 0 / 1e-4 / 1e-3) with the
  oracle's hit flags and time-of-impact intervals.

Run from the repository root:  python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import pyoracle  # noqa: E402
from silk_physics_b200 import native as N  # noqa: E402
from silk_physics_b200 import scenes as S  # noqa: E402

C1_STEPS = (1, 5, 10)
C1_CONFIG = dict(max_inner_iteration=10, admm_abs_tol=0.0, admm_rel_tol=0.0,
                 fixed_linear_rel_tol=1e-6)
CCD_ERR = {True: 4.053116e-06, False: 3.814698e-06}


# (is_collision_on, is_self_collision_on, group, restitution, friction)
C1_COLLISION = {False: (0, 0, 0, 0.3, 0.3), True: (1, 1, 0, 0.3, 0.3)}


def c1_sheet(self_collision=False):
    V, F = S.grid_sheet(32, jitter=0.0, seed=7)
    P = S.top_corner_pins(32)
    perm, offs = N.partition_mesh(V, F)
    out = {"verts": V, "faces": F, "pins": P, "perm": perm, "part_offsets": offs}
    for name, fp64 in (("o64", True), ("o32", False)):
        ow = pyoracle.OracleWorld(fp64=fp64, config=C1_CONFIG)
        h = ow.add_cloth(V, F, P, perm, offs, collision=C1_COLLISION[self_collision])
        for k in range(1, max(C1_STEPS) + 1):
            assert ow.step() == 0
            if k in C1_STEPS:
                out[f"{name}_step{k}"] = ow.position(h)
                if self_collision:
                    out[f"{name}_contacts{k}"] = np.int32(ow.stats()["contacts"])
    return out


def ccd_queries(vf, n=256):
    rng = np.random.default_rng(4242 if vf else 4243)
    base = rng.uniform(-1, 1, (n, 4, 3)).astype(np.float32)
    if vf:
        base[:, 1:, 2] = 0.0
        base[:, 0, 2] = rng.uniform(0.001, 0.2, n)
    motion = rng.normal(0, 0.4, (n, 4, 3)).astype(np.float32)
    motion[:, 0, 2] -= rng.uniform(0, 0.6, n)
    x = np.concatenate([base, base + motion], axis=1).reshape(n, 24).astype(np.float32)
    ms = rng.choice([0.0, 1e-4, 1e-3], n).astype(np.float32)
    err = np.full(3, CCD_ERR[vf], np.float32)
    hit = np.zeros(n, np.int32)
    toi = np.zeros(n, np.float32)
    tup = np.zeros(n, np.float32)
    for i in range(n):
        h, t4, small = pyoracle.ccd(vf, x[i], err, float(ms[i]))
        hit[i] = int(h)
        if h:
            toi[i] = t4[2] if small else t4[0]
            tup[i] = t4[3] if small else t4[1]
    return x, ms, hit, toi, tup


def main():
    pyoracle.build()
    np.savez_compressed(HERE / "c1_sheet32.npz", **c1_sheet())
    np.savez_compressed(HERE / "c1_sheet32_selfcol.npz", **c1_sheet(self_collision=True))
    out = {}
    for vf, tag in ((True, "vf"), (False, "ee")):
        x, ms, hit, toi, tup = ccd_queries(vf)
        out.update({f"{tag}_x": x, f"{tag}_ms": ms, f"{tag}_hit": hit, f"{tag}_toi": toi,
                    f"{tag}_tup": tup})
    np.savez_compressed(HERE / "ccd_queries.npz", **out)
    print("written", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
