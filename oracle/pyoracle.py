"""ctypes wrapper of the CPU oracle (oracle/build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "liboracle.so"
# The reference's own CPU CCD (silk/src/backend/cpu/collision/ccd.cpp,
# interval_root_finder.cpp, interval.cpp) compiled unchanged by `make ref`
# where the reference checkout is present; the built library travels with
# the tree.
REF_LIB = HERE / "_ref" / "libref_ccd.so"
REF_CHECKOUT = Path("/root/reference")


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if (REF_CHECKOUT / "silk" / "src" / "backend" / "cpu" / "collision" / "ccd.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REF_CHECKOUT}"], check=True)
    return LIB


class GlobalConfig(C.Structure):
    _fields_ = [("acceleration", C.c_float * 3), ("max_outer_iteration", C.c_int),
                ("max_inner_iteration", C.c_int), ("dt", C.c_float),
                ("linear_solver_abs_tol", C.c_float), ("linear_solver_rel_tol_min", C.c_float),
                ("linear_solver_rel_tol_max", C.c_float), ("initial_linear_rel_tol", C.c_float),
                ("admm_abs_tol", C.c_float), ("admm_rel_tol", C.c_float),
                ("fixed_linear_rel_tol", C.c_float), ("cg_max_iter", C.c_int)]


class ClothConfig(C.Structure):
    _fields_ = [("elastic_stiffness", C.c_float), ("bending_stiffness", C.c_float),
                ("density", C.c_float), ("damping", C.c_float)]


class CollisionConfig(C.Structure):
    _fields_ = [("is_collision_on", C.c_int), ("is_self_collision_on", C.c_int),
                ("group", C.c_int), ("restitution", C.c_float), ("friction", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("outer_iterations", C.c_int), ("admm_iterations", C.c_int),
                ("cg_iterations", C.c_int), ("cg_solves", C.c_int), ("contacts", C.c_int),
                ("colors", C.c_int), ("ccd_queries", C.c_int), ("ccd_hits", C.c_int),
                ("min_toi", C.c_float)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _lib.oracle_world_new.restype = C.c_void_p
        _lib.oracle_world_new.argtypes = [C.c_int]
        _lib.oracle_world_free.argtypes = [C.c_void_p]
        _lib.oracle_debug_min_toi.restype = C.c_float
        _lib.oracle_debug_min_toi.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float,
                                             C.POINTER(C.c_int), C.POINTER(C.c_int)]
        for name in ["oracle_set_global_config", "oracle_add_cloth", "oracle_add_obstacle",
                     "oracle_set_obstacle_position", "oracle_set_cloth_pin_position",
                     "oracle_solver_step", "oracle_get_cloth_position",
                     "oracle_get_cloth_position_f64", "oracle_get_stats",
                     "oracle_cloth_dense_scalar_matrix", "oracle_cloth_dense_full_matrix",
                     "oracle_cloth_vectors", "oracle_debug_candidates", "oracle_debug_refit",
                     "oracle_debug_dcd", "oracle_set_cloth_state"]:
            getattr(_lib, name).restype = C.c_int
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleWorld:
    """CPU restatement of one silk::World (FP32 or FP64 solver arithmetic)."""

    def __init__(self, fp64: bool = False, config: dict | None = None):
        self.L = lib()
        self.w = C.c_void_p(self.L.oracle_world_new(int(fp64)))
        self.nv: dict[int, int] = {}
        g = GlobalConfig()
        cfg = dict(acceleration=(0.0, 0.0, -10.0), max_outer_iteration=100,
                   max_inner_iteration=100, dt=1.0 / 60.0, linear_solver_abs_tol=1e-7,
                   linear_solver_rel_tol_min=1e-6, linear_solver_rel_tol_max=1e-3,
                   initial_linear_rel_tol=1e-2, admm_abs_tol=1e-5, admm_rel_tol=1e-3,
                   fixed_linear_rel_tol=0.0, cg_max_iter=1000)
        cfg.update(config or {})
        for k, v in cfg.items():
            if k == "acceleration":
                g.acceleration = (C.c_float * 3)(*v)
            else:
                setattr(g, k, v)
        self.L.oracle_set_global_config(self.w, C.byref(g))

    def __del__(self):
        if getattr(self, "w", None):
            self.L.oracle_world_free(self.w)
            self.w = None

    def add_cloth(self, verts, faces, pins, perm, part_offsets, cloth=None, collision=None):
        cc = ClothConfig(*(cloth or (100.0, 1e-4, 0.1, 0.01)))
        col = CollisionConfig(*(collision or (1, 1, 0, 0.3, 0.3)))
        v = np.ascontiguousarray(verts, np.float32).ravel()
        f = np.ascontiguousarray(faces, np.int32).ravel()
        p = np.ascontiguousarray(pins, np.int32).ravel()
        pm = np.ascontiguousarray(perm, np.int32).ravel()
        po = np.ascontiguousarray(part_offsets, np.int32).ravel()
        h = C.c_uint32(0)
        st = self.L.oracle_add_cloth(self.w, C.byref(cc), C.byref(col), _p(v, C.c_float),
                                     v.size // 3, _p(f, C.c_int), f.size // 3, _p(p, C.c_int),
                                     p.size, _p(pm, C.c_int), _p(po, C.c_int), po.size - 1,
                                     C.byref(h))
        assert st == 0
        self.nv[h.value] = v.size // 3
        return h.value

    def add_obstacle(self, verts, faces, collision=None):
        col = CollisionConfig(*(collision or (1, 1, 0, 0.3, 0.3)))
        v = np.ascontiguousarray(verts, np.float32).ravel()
        f = np.ascontiguousarray(faces, np.int32).ravel()
        h = C.c_uint32(0)
        st = self.L.oracle_add_obstacle(self.w, C.byref(col), _p(v, C.c_float), v.size // 3,
                                        _p(f, C.c_int), f.size // 3, C.byref(h))
        assert st == 0
        return h.value

    def set_obstacle_position(self, h, pos):
        p = np.ascontiguousarray(pos, np.float32).ravel()
        return self.L.oracle_set_obstacle_position(self.w, h, _p(p, C.c_float), p.size)

    def set_cloth_pin_position(self, h, pos):
        p = np.ascontiguousarray(pos, np.float32).ravel()
        return self.L.oracle_set_cloth_pin_position(self.w, h, _p(p, C.c_float), p.size)

    def step(self) -> int:
        return self.L.oracle_solver_step(self.w)

    def set_state(self, h, x, v):
        xs = np.ascontiguousarray(x, np.float32).ravel()
        vs = np.ascontiguousarray(v, np.float32).ravel()
        return self.L.oracle_set_cloth_state(self.w, h, _p(xs, C.c_float), _p(vs, C.c_float),
                                             xs.size)

    def position_f32(self, h) -> np.ndarray:
        out = np.zeros(3 * self.nv[h], np.float32)
        assert self.L.oracle_get_cloth_position(self.w, h, _p(out, C.c_float), out.size) == 0
        return out.reshape(-1, 3)

    def velocity(self, h) -> np.ndarray:
        out = np.zeros(3 * self.nv[h], np.float32)
        assert self.L.oracle_get_cloth_velocity(self.w, h, _p(out, C.c_float), out.size) == 0
        return out.reshape(-1, 3)

    def position(self, h) -> np.ndarray:
        out = np.zeros(3 * self.nv[h], np.float64)
        assert self.L.oracle_get_cloth_position_f64(self.w, h, _p(out, C.c_double),
                                                    out.size) == 0
        return out.reshape(-1, 3)

    def stats(self) -> dict:
        s = Stats()
        self.L.oracle_get_stats(self.w, C.byref(s))
        return {n: getattr(s, n) for n, _ in Stats._fields_}

    def scalar_matrix(self, h) -> np.ndarray:
        n = self.nv[h]
        out = np.zeros(n * n, np.float64)
        assert self.L.oracle_cloth_dense_scalar_matrix(self.w, h, _p(out, C.c_double), n) == 0
        return out.reshape(n, n)

    def full_matrix(self, h) -> np.ndarray:
        n = 3 * self.nv[h]
        out = np.zeros(n * n, np.float64)
        assert self.L.oracle_cloth_dense_full_matrix(self.w, h, _p(out, C.c_double), n) == 0
        return out.reshape(n, n)

    def vectors(self, h):
        n = 3 * self.nv[h]
        m, cw, br = (np.zeros(n, np.float64) for _ in range(3))
        assert self.L.oracle_cloth_vectors(self.w, h, _p(m, C.c_double), _p(cw, C.c_double),
                                           _p(br, C.c_double), n) == 0
        return m, cw, br

    def refit(self, disp=None):
        if disp is None:
            self.L.oracle_debug_refit(self.w, None, 0)
        else:
            d = np.ascontiguousarray(disp, np.float32).ravel()
            self.L.oracle_debug_refit(self.w, _p(d, C.c_float), d.size)

    def candidates(self, cap=1 << 22) -> np.ndarray:
        out = np.zeros(5 * cap, np.int32)
        n = self.L.oracle_debug_candidates(self.w, _p(out, C.c_int), cap)
        return out[: 5 * min(n, cap)].reshape(-1, 5)

    def dcd(self, t, dact, cap=1 << 20) -> np.ndarray:
        out = np.zeros(7 * cap, np.int32)
        n = self.L.oracle_debug_dcd(self.w, C.c_float(t), C.c_float(dact), _p(out, C.c_int),
                                    cap)
        return out[: 7 * min(n, cap)].reshape(-1, 7)

    def min_toi(self, ts, mt, ms):
        nq, nh = C.c_int(0), C.c_int(0)
        t = self.L.oracle_debug_min_toi(self.w, ts, mt, ms, C.byref(nq), C.byref(nh))
        return t, nq.value, nh.value


def ccd(is_vf: bool, x24, err3, ms, tol=1e-6, max_iter=4096, no_zero_toi=True,
        max_time=1.0):
    L = lib()
    x = np.ascontiguousarray(x24, np.float32).ravel()
    e = np.ascontiguousarray(err3, np.float32).ravel()
    t4 = np.zeros(4, np.float32)
    small = C.c_int(0)
    hit = L.oracle_ccd(int(is_vf), _p(x, C.c_float), _p(e, C.c_float), C.c_float(ms),
                       C.c_float(tol), C.c_long(max_iter), int(no_zero_toi),
                       C.c_float(max_time), _p(t4, C.c_float), C.byref(small))
    return bool(hit), t4, bool(small.value)


def ccd_toi(is_vf, x24, err3, ms, tol=1e-6, max_iter=4096, max_time=1.0):
    """Time of impact as the production step consumes it."""
    hit, t4, small = ccd(is_vf, x24, err3, ms, tol, max_iter, True, max_time)
    if not hit:
        return False, max_time
    return True, float(t4[2] if small else t4[0])


def color_contacts(verts4, prio):
    L = lib()
    v = np.ascontiguousarray(verts4, np.int32).ravel()
    p = np.ascontiguousarray(prio, np.uint64).ravel()
    out = np.zeros(p.size, np.int32)
    nc = L.oracle_color_contacts(_p(v, C.c_int), _p(p, C.c_uint64), p.size, _p(out, C.c_int))
    return out, nc


_ref_lib = None


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib() -> C.CDLL:
    """The reference's own CCD (oracle/_ref/libref_ccd.so)."""
    global _ref_lib
    if _ref_lib is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle ref)")
        _ref_lib = C.CDLL(str(REF_LIB))
        _ref_lib.ref_ccd.restype = C.c_int
        _ref_lib.ref_ccd.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                     C.c_float, C.c_float, C.c_long, C.c_int, C.c_float,
                                     C.POINTER(C.c_float), C.POINTER(C.c_int),
                                     C.POINTER(C.c_float)]
        _ref_lib.ref_numerical_error.restype = None
    return _ref_lib


def ref_ccd(is_vf: bool, x24, err3, ms, tol=1e-6, max_iter=4096, no_zero_toi=True,
            max_time=1.0):
    """silk::cpu::vertex_face_ccd / edge_edge_ccd of the reference itself:
    (hit, t4 = [t_lo, t_hi, small_ms_t_lo, small_ms_t_hi], use_small_ms,
    tolerance)."""
    L = ref_lib()
    x = np.ascontiguousarray(x24, np.float32).ravel()
    e = np.ascontiguousarray(err3, np.float32).ravel()
    t4 = np.zeros(4, np.float32)
    small = C.c_int(0)
    tolr = C.c_float(0.0)
    hit = L.ref_ccd(int(is_vf), _p(x, C.c_float), _p(e, C.c_float), C.c_float(ms),
                    C.c_float(tol), C.c_long(max_iter), int(no_zero_toi), C.c_float(max_time),
                    _p(t4, C.c_float), C.byref(small), C.byref(tolr))
    return bool(hit), t4, bool(small.value), float(tolr.value)


def ref_ccd_toi(is_vf, x24, err3, ms, tol=1e-6, max_iter=4096, max_time=1.0):
    """The reference's answer as the solver step consumes it: (hit, toi,
    t_upper) from the accepted interval, or from the refined-separation
    interval when the first starts at 0 (ccd.cpp:150-180 with
    narrowphase.cu:66)."""
    hit, t4, small, _ = ref_ccd(is_vf, x24, err3, ms, tol, max_iter, True, max_time)
    if not hit:
        return False, max_time, max_time
    return True, float(t4[2] if small else t4[0]), float(t4[3] if small else t4[1])


def ref_numerical_error(absmax3, is_vf: bool) -> np.ndarray:
    L = ref_lib()
    a = np.ascontiguousarray(absmax3, np.float32).ravel()
    out = np.zeros(3, np.float32)
    L.ref_numerical_error(_p(a, C.c_float), int(is_vf), _p(out, C.c_float))
    return out
