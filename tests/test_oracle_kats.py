"""The oracle pinned against the reference's own known-answer tests."""
import ctypes as C
from fractions import Fraction

import numpy as np
import pytest


def _coulomb(oracle, u, n, mu):
    L = oracle.lib()
    f3 = C.c_float * 3
    out = f3()
    L.oracle_solve_coulomb(f3(*u), f3(*n), C.c_float(mu), out)
    return np.array(list(out), np.float32)


def test_exact_ee_uv_crossing_edges(oracle):
    """test/friction_contact_test.cu:10-21."""
    L = oracle.lib()
    x = (C.c_float * 12)(-0.005, 0, 0, 0.005, 0, 0, 0, -0.005, 0.0005, 0, 0.005, 0.0005)
    uv = (C.c_float * 2)()
    assert L.oracle_exact_ee_uv(x, C.c_float(1e-6), uv) == 1
    assert uv[0] == pytest.approx(0.5) and uv[1] == pytest.approx(0.5)


def test_coulomb_known_answers(oracle):
    """test/friction_contact_test.cu:23-63."""
    n = (0.0, 0.0, 1.0)
    assert _coulomb(oracle, (1, -2, 0.5), n, 0.7).tolist() == [1.0, -2.0, 0.5]
    assert _coulomb(oracle, (0.2, 0, -1), n, 0.5).tolist() == [0.0, 0.0, 0.0]
    assert _coulomb(oracle, (2, 0, -1), n, 0.5).tolist() == [1.5, 0.0, 0.0]
    assert _coulomb(oracle, (2, -3, -1), n, 0.0).tolist() == [2.0, -3.0, 0.0]


def test_coulomb_complementarity_and_cone(oracle):
    """test/friction_contact_test.cu:65-92."""
    n = np.array([0, 0, 1.0], np.float32)
    for mu in [0.0, 0.1, 0.5, 2.0]:
        for u in [(0, 0, 1), (2, -1, 0), (0.1, 0.2, -1), (2, 0, -1), (-3, 4, -0.5),
                  (0, 0, -2)]:
            s = _coulomb(oracle, u, n, mu)
            r = s - np.array(u, np.float32)
            sn, rn = s @ n, r @ n
            rt = r - rn * n
            assert sn >= -1e-5 and rn >= -1e-5
            assert abs(sn * rn) <= 1e-5
            assert np.linalg.norm(rt) <= mu * rn + 1e-5


def test_numerical_filter_constants(oracle):
    """interval_root_finder.cpp:512-522 from the derivation in
    test/narrowphase/derive_numerical_filter.py: EE = 32 eps, VF = 34 eps with
    eps = 2^-23, scaled by max(|x|, 1) per axis."""
    L = oracle.lib()
    eps = Fraction(1, 2 ** 23)
    ee, vf = float(32 * eps), float(34 * eps)
    # The reference constants are the derived bounds rounded up in decimal.
    for derived, const in ((ee, 3.814698e-06), (vf, 4.053116e-06)):
        assert np.float32(const) >= np.float32(derived)
        assert abs(float(np.float32(const)) - derived) / derived < 1e-6
    out = (C.c_float * 3)()
    L.oracle_numerical_error((C.c_float * 3)(0.5, 2.0, 3.0), 1, out)
    assert list(out) == [np.float32(4.053116e-06), np.float32(4.053116e-06) * np.float32(2.0),
                         np.float32(4.053116e-06) * np.float32(3.0)]


def test_ccd_simple_cases(oracle):
    err = [4.053116e-06] * 3
    # Point falling through a triangle at t = 0.5 (z from 1 to -1).
    x = np.array([[0.2, 0.2, 1], [0, 0, 0], [1, 0, 0], [0, 1, 0],
                  [0.2, 0.2, -1], [0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    hit, t4, small = oracle.ccd(True, x, err, 0.0)
    assert hit and abs(t4[0] - 0.5) < 1e-5 and t4[0] <= 0.5
    # Point passing beside the triangle: no hit.
    x2 = x.copy()
    x2[[0, 4], 0] = 3.0
    assert not oracle.ccd(True, x2, err, 0.0)[0]
    # Edge-edge crossing at t = 0.25.
    e = np.array([[-1, 0, 0.25], [1, 0, 0.25], [0, -1, 0], [0, 1, 0],
                  [-1, 0, -0.75], [1, 0, -0.75], [0, -1, 0], [0, 1, 0]], np.float32)
    hit, t4, _ = oracle.ccd(False, e, [3.814698e-06] * 3, 0.0)
    assert hit and abs(t4[0] - 0.25) < 1e-5
    # Minimum separation: a point resting at distance 1e-3 with ms = 2e-3 hits
    # at t = 0, the refined ms = 1e-3 then reports the full interval.
    x3 = np.array([[0.2, 0.2, 1e-3], [0, 0, 0], [1, 0, 0], [0, 1, 0],
                   [0.2, 0.2, 1e-3], [0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    hit, t4, small = oracle.ccd(True, x3, err, 2e-3)
    assert hit and t4[0] == 0.0 and small


def test_greedy_coloring_is_valid(oracle):
    rng = np.random.default_rng(5)
    verts = rng.integers(-1, 40, size=(300, 4)).astype(np.int32)
    prio = rng.integers(0, 2 ** 63, size=300, dtype=np.uint64)
    colors, nc = oracle.color_contacts(verts, prio)
    assert colors.min() >= 1 and colors.max() == nc
    for i in range(300):
        for j in range(i + 1, 300):
            a = set(verts[i][verts[i] >= 0]) & set(verts[j][verts[j] >= 0])
            if a:
                assert colors[i] != colors[j]


def test_touching_boxes_are_candidates(oracle):
    """test/broadphase/main.cpp:353-380: boxes that share a face overlap."""
    from silk_physics_b200 import scenes as S

    # Two cloth sheets whose padded boxes touch exactly along z.
    V, F = S.grid_sheet(3, side=1.0, z=0.0)
    ow = oracle.OracleWorld()
    perm = np.arange(len(V), dtype=np.int32)
    offs = np.array([0, len(V)], np.int32)
    ow.add_cloth(V, F, [], perm, offs, collision=(1, 0, 0, 0.3, 0.3))
    pad = 0.05 * 0.5 * (1 + 2 ** 0.5 * 2 / 3)  # not needed exactly; see below
    del pad
    V2 = V.copy()
    ow.add_cloth(V2, F, [], perm, offs, collision=(1, 0, 0, 0.3, 0.3))
    ow.refit()
    c = ow.candidates()
    assert len(c) > 0


def test_reference_arm_state_file():
    """The stored oracle state the reference arm of bench.py starts from:
    the 80x80 benchmark sheet after 27 steps, finite, in contact range of
    the sphere (z of the lowest vertex near its top at 0.3 m)."""
    from pathlib import Path

    import numpy as np

    st = np.load(Path(__file__).resolve().parent.parent / "oracle" /
                 "reference_state_c2_step27.npz")
    assert int(st["steps"]) == 27
    assert st["x"].shape == (6400, 3) and st["v"].shape == (6400, 3)
    assert np.isfinite(st["x"]).all() and np.isfinite(st["v"]).all()
    assert 0.0 < st["x"][:, 2].min() < 0.6
