"""ctypes binding of libsilk_b200.so and the Python ``World`` mirror."""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libsilk_b200.so"


class ErrorCode(enum.IntEnum):
    """silk::ErrorCode (silk/include/silk/result.hpp:22-35)."""

    Unknown = 0
    NotInitialized = 1
    InvalidConfig = 2
    TooManyBody = 3
    InvalidHandle = 4
    InvalidMesh = 5
    InvalidPin = 6
    InvalidPosition = 7
    CholeskyDecompositionFail = 8
    NeedInitSolverFirst = 9
    IterativeSolveFail = 10
    NoCudaSupport = 11


class Backend(enum.IntEnum):
    CPU = 0
    GPU = 1


@dataclass
class Result:
    """silk::Result: truthy on success; ``code`` and ``detail`` on error."""

    success: bool = True
    code: ErrorCode = ErrorCode.Unknown
    detail: str = ""

    def __bool__(self) -> bool:
        return self.success

    def to_string(self) -> str:
        if self.success:
            return "OK"
        if not self.detail:
            return self.code.name
        return f"{self.code.name}. Reason: {self.detail}."


class _GlobalConfigC(C.Structure):
    _fields_ = [
        ("acceleration_x", C.c_float), ("acceleration_y", C.c_float),
        ("acceleration_z", C.c_float), ("max_outer_iteration", C.c_int32),
        ("max_inner_iteration", C.c_int32), ("dt", C.c_float),
        ("linear_solver_abs_tol", C.c_float), ("linear_solver_rel_tol_min", C.c_float),
        ("linear_solver_rel_tol_max", C.c_float), ("initial_linear_rel_tol", C.c_float),
        ("admm_abs_tol", C.c_float), ("admm_rel_tol", C.c_float),
    ]


class _ClothConfigC(C.Structure):
    _fields_ = [("elastic_stiffness", C.c_float), ("bending_stiffness", C.c_float),
                ("density", C.c_float), ("damping", C.c_float)]


class _CollisionConfigC(C.Structure):
    _fields_ = [("is_collision_on", C.c_int32), ("is_self_collision_on", C.c_int32),
                ("group", C.c_int32), ("restitution", C.c_float), ("friction", C.c_float)]


class _SolverOptionsC(C.Structure):
    _fields_ = [("fixed_linear_rel_tol", C.c_float), ("cg_max_iter", C.c_int32),
                ("mas_bf16", C.c_int32), ("profile", C.c_int32), ("cg_form", C.c_int32),
                ("learned_warm_start", C.c_int32), ("capture_samples", C.c_int32),
                ("contact_gs_form", C.c_int32), ("admm_extrapolated_start", C.c_int32),
                ("resident_halo_limit", C.c_int32), ("barrier_spin_limit", C.c_int32),
                ("debug_withhold_block", C.c_int32), ("admm_check_interval", C.c_int32)]


class _ProfileC(C.Structure):
    _fields_ = [("cg_time_ms", C.c_double), ("cg_launches", C.c_int64),
                ("cg_iterations", C.c_int64), ("cg_algorithmic_bytes", C.c_double),
                ("admm_other_ms", C.c_double), ("admm_host_ms", C.c_double),
                ("ccd_host_ms", C.c_double), ("dcd_host_ms", C.c_double),
                ("step_host_ms", C.c_double), ("contact_gs_ms", C.c_double),
                ("ccd_refit_host_ms", C.c_double), ("ccd_candidates_host_ms", C.c_double),
                ("ccd_first_pass_ms", C.c_double), ("ccd_second_pass_ms", C.c_double),
                ("ccd_second_pass_queries", C.c_double), ("ccd_calls", C.c_double),
                ("dcd_refit_host_ms", C.c_double), ("dcd_candidates_host_ms", C.c_double),
                ("dcd_build_host_ms", C.c_double), ("dcd_coloring_host_ms", C.c_double),
                ("dcd_layout_host_ms", C.c_double), ("dcd_calls", C.c_double)]


class _StepStatsC(C.Structure):
    _fields_ = [("outer_iterations", C.c_int32), ("admm_iterations", C.c_int32),
                ("cg_iterations", C.c_int32), ("cg_solves", C.c_int32),
                ("contacts", C.c_int32), ("colors", C.c_int32),
                ("ccd_queries", C.c_int32), ("ccd_hits", C.c_int32),
                ("min_toi", C.c_float), ("broadphase_candidates", C.c_int32),
                ("kernel_launches", C.c_int64), ("cg_resident_solves", C.c_int32),
                ("cg_first_solve_iterations", C.c_int32), ("learned_starts", C.c_int32),
                ("extrapolated_starts", C.c_int32), ("cg_cluster_solves", C.c_int32),
                ("learned_iterate_starts", C.c_int32)]


@dataclass
class GlobalConfig:
    """silk::GlobalConfig (silk.hpp:47-77)."""

    acceleration_x: float = 0.0
    acceleration_y: float = 0.0
    acceleration_z: float = -10.0
    max_outer_iteration: int = 100
    max_inner_iteration: int = 100
    dt: float = 1.0 / 60.0
    linear_solver_abs_tol: float = 1e-7
    linear_solver_rel_tol_min: float = 1e-6
    linear_solver_rel_tol_max: float = 1e-3
    initial_linear_rel_tol: float = 1e-2
    admm_abs_tol: float = 1e-5
    admm_rel_tol: float = 1e-3

    def to_c(self) -> _GlobalConfigC:
        return _GlobalConfigC(*[getattr(self, n) for n, _ in _GlobalConfigC._fields_])


@dataclass
class ClothConfig:
    """silk::ClothConfig (silk.hpp:35-45)."""

    elastic_stiffness: float = 100.0
    bending_stiffness: float = 0.0001
    density: float = 0.1
    damping: float = 0.01

    def to_c(self) -> _ClothConfigC:
        return _ClothConfigC(self.elastic_stiffness, self.bending_stiffness,
                             self.density, self.damping)


@dataclass
class CollisionConfig:
    """silk::CollisionConfig (silk.hpp:26-33)."""

    is_collision_on: bool = True
    is_self_collision_on: bool = True
    group: int = 0
    restitution: float = 0.3
    friction: float = 0.3

    def to_c(self) -> _CollisionConfigC:
        return _CollisionConfigC(int(self.is_collision_on), int(self.is_self_collision_on),
                                 self.group, self.restitution, self.friction)


@dataclass
class SolverOptions:
    """Switches with no silk::GlobalConfig field (bench / precision modes)."""

    fixed_linear_rel_tol: float = 0.0
    cg_max_iter: int = 1000
    mas_bf16: bool = False
    profile: int = 0  # 1: CUDA-event kernel timing; 2: also the CG phase trace
    cg_form: int = 0  # 0: cluster form, else resident, else streaming; 2: no cluster form; 1: streaming; 3/4: as 0/2 with the rows in global memory
    learned_warm_start: bool = False  # offer the loaded model's first-solve start
    capture_samples: int = 0  # bit 1: first-solve samples, bit 2: iterate-model samples
    contact_gs_form: int = 0          # 0: single-block Gauss-Seidel where possible; 1: grid
    admm_extrapolated_start: bool = False  # offer 2 x_k - x_(k-1) as later CG starts
    resident_halo_limit: int = 0  # > 0: fewer halo slots per resident-CG block (0: 1024)
    barrier_spin_limit: int = 0  # > 0: polls before a CG grid-barrier wait gives up
    debug_withhold_block: int = 0  # k > 0: block k - 1 of a cooperative CG grid never arrives
    admm_check_interval: int = 0  # ADMM iterations between host reads of the device's convergence state (0: 4)

    def to_c(self) -> _SolverOptionsC:
        o = _SolverOptionsC()
        o.fixed_linear_rel_tol = self.fixed_linear_rel_tol
        o.cg_max_iter = self.cg_max_iter
        o.mas_bf16 = int(self.mas_bf16)
        o.profile = int(self.profile)
        o.cg_form = int(self.cg_form)
        o.learned_warm_start = int(self.learned_warm_start)
        o.capture_samples = int(self.capture_samples)
        o.contact_gs_form = int(self.contact_gs_form)
        o.admm_extrapolated_start = int(self.admm_extrapolated_start)
        o.resident_halo_limit = int(self.resident_halo_limit)
        o.barrier_spin_limit = int(self.barrier_spin_limit)
        o.debug_withhold_block = int(self.debug_withhold_block)
        o.admm_check_interval = int(self.admm_check_interval)
        return o


@dataclass
class StepStats:
    outer_iterations: int = 0
    admm_iterations: int = 0
    cg_iterations: int = 0
    cg_solves: int = 0
    contacts: int = 0
    colors: int = 0
    ccd_queries: int = 0
    ccd_hits: int = 0
    min_toi: float = 0.0
    broadphase_candidates: int = 0
    kernel_launches: int = 0
    cg_resident_solves: int = 0
    cg_first_solve_iterations: int = 0
    learned_starts: int = 0
    extrapolated_starts: int = 0
    cg_cluster_solves: int = 0
    learned_iterate_starts: int = 0


_F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_U64P = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_W = C.c_void_p


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -m silk_physics_b200.build`")
    L = C.CDLL(str(_LIB_PATH))
    sig = {
        "silk_world_create": ([], _W),
        "silk_world_destroy": ([_W], None),
        "silk_world_last_error": ([_W], C.c_char_p),
        "silk_world_init": ([_W, C.c_int32], C.c_int),
        "silk_set_global_config": ([_W, C.POINTER(_GlobalConfigC)], C.c_int),
        "silk_global_config_default": ([C.POINTER(_GlobalConfigC)], None),
        "silk_clear": ([_W], None),
        "silk_solver_step": ([_W], C.c_int),
        "silk_solver_reset": ([_W], C.c_int),
        "silk_step_many": ([C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(C.c_int)],
                           C.c_int),
        "silk_add_cloth": ([_W, C.POINTER(_ClothConfigC), C.POINTER(_CollisionConfigC),
                            _F32P, C.c_int64, _I32P, C.c_int64, C.c_void_p, C.c_int64,
                            C.POINTER(C.c_uint32)], C.c_int),
        "silk_remove_cloth": ([_W, C.c_uint32], C.c_int),
        "silk_get_cloth_position": ([_W, C.c_uint32, _F32P, C.c_int64], C.c_int),
        "silk_set_cloth_config": ([_W, C.c_uint32, C.POINTER(_ClothConfigC)], C.c_int),
        "silk_set_cloth_collision_config": ([_W, C.c_uint32, C.POINTER(_CollisionConfigC)],
                                            C.c_int),
        "silk_set_cloth_pin_index": ([_W, C.c_uint32, C.c_void_p, C.c_int64], C.c_int),
        "silk_set_cloth_pin_position": ([_W, C.c_uint32, C.c_void_p, C.c_int64], C.c_int),
        "silk_add_obstacle": ([_W, C.POINTER(_CollisionConfigC), _F32P, C.c_int64, C.c_void_p,
                               C.c_int64, C.POINTER(C.c_uint32)], C.c_int),
        "silk_remove_obstacle": ([_W, C.c_uint32], C.c_int),
        "silk_set_obstacle_collision_config": ([_W, C.c_uint32,
                                                C.POINTER(_CollisionConfigC)], C.c_int),
        "silk_set_obstacle_position": ([_W, C.c_uint32, _F32P, C.c_int64], C.c_int),
        "silk_solver_options_default": ([C.POINTER(_SolverOptionsC)], None),
        "silk_set_solver_options": ([_W, C.POINTER(_SolverOptionsC)], C.c_int),
        "silk_get_step_stats": ([_W, C.POINTER(_StepStatsC)], C.c_int),
        "silk_set_stream": ([_W, C.c_void_p], C.c_int),
        "silk_get_profile": ([_W, C.POINTER(_ProfileC), C.c_int32], C.c_int),
        "silk_get_cloth_velocity": ([_W, C.c_uint32, _F32P, C.c_int64], C.c_int),
        "silk_set_cloth_state": ([_W, C.c_uint32, _F32P, C.c_int64, C.c_void_p, C.c_int64],
                                 C.c_int),
        "silk_debug_coulomb": ([_F32P, _F32P, _F32P, C.c_int64, _F32P], C.c_int),
        "silk_debug_cloth_partition": ([_W, C.c_uint32, _I32P, C.c_int64, _I32P, C.c_int64,
                                        C.POINTER(C.c_int32)], C.c_int),
        "silk_debug_cloth_matrix": ([_W, C.c_uint32, _F64P, C.c_int64], C.c_int),
        "silk_debug_refit": ([_W, C.c_void_p, C.c_int64], C.c_int),
        "silk_debug_candidates": ([_W, _I32P, C.c_int64, C.POINTER(C.c_int32)], C.c_int),
        "silk_debug_dcd": ([_W, C.c_float, C.c_float, _I32P, C.c_int64,
                            C.POINTER(C.c_int32)], C.c_int),
        "silk_debug_cg_trace": ([_W, C.c_uint32, C.c_void_p, C.c_int64, C.POINTER(C.c_int32)],
                                C.c_int),
        "silk_debug_contacts": ([_W, _I32P, C.c_int64, C.POINTER(C.c_int32)], C.c_int),
        "silk_debug_min_toi": ([_W, C.c_float, C.c_float, C.c_float, C.c_int32,
                                C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32)], C.c_int),
        "silk_ccd_batch": ([C.c_int32, _F32P, C.c_int64, _F32P, _F32P, C.c_float, C.c_int32,
                            C.c_float, _I32P, _F32P, _F32P], C.c_int),
        "silk_color_contacts": ([_I32P, _U64P, C.c_int64, _I32P, C.POINTER(C.c_int32)],
                                C.c_int),
        "silk_set_warm_start_model": ([_W, C.c_void_p, C.c_int64], C.c_int),
        "silk_get_iterate_samples": ([_W, _F32P, _F32P, C.c_int64, C.POINTER(C.c_int32)],
                                     C.c_int),
        "silk_get_warm_start_samples": ([_W, C.c_uint32, _F32P, _F32P, C.c_int64,
                                         C.POINTER(C.c_int32)], C.c_int),
        "silk_mlp_forward": ([_F32P, _F32P, C.c_int64, _F32P], C.c_int),
        "silk_mlp_loss_grad": ([_F32P, _F32P, _F32P, C.c_int64, _F32P,
                                C.POINTER(C.c_double)], C.c_int),
        "silk_mlp_train": ([_F32P, _F32P, _F32P, C.c_int64, C.c_int32, C.c_int32, C.c_float,
                            C.c_uint64, C.c_void_p], C.c_int),
        "silk_ccd_batch_noalloc": ([C.c_int32, C.c_void_p, C.c_int64, _F32P, C.c_void_p,
                                    C.c_float, C.c_int32, C.c_float, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)], C.c_int),
        "silk_debug_mas_fine": ([_W, C.c_uint32, _F32P, C.c_int64, _F32P, C.c_int64], C.c_int),
        "silk_partition_mesh": ([_F32P, C.c_int64, _I32P, C.c_int64, _I32P, _I32P, C.c_int64,
                                 C.POINTER(C.c_int32)], C.c_int),
        "silk_schedule_bank_rows": ([_I32P, _I32P, _I32P, C.c_int32, C.c_int32, _I32P, _I32P],
                                    C.c_int),
        "silk_assemble_cloth_host": ([C.POINTER(_ClothConfigC), _F32P, C.c_int64, _I32P,
                                      C.c_int64, C.c_float, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


lib = _load()


def _result(status: int, world=None) -> Result:
    if status == 0:
        return Result()
    detail = ""
    if world is not None:
        detail = (lib.silk_world_last_error(world) or b"").decode()
    return Result(False, ErrorCode(status - 1), detail)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


class World:
    """Python mirror of silk::World (silk.hpp:83-239).

    Methods return ``Result``; ``add_cloth`` / ``add_obstacle`` return a
    ``(Result, handle)`` pair because Python has no out-references.
    """

    def __init__(self) -> None:
        self._w = lib.silk_world_create()
        if not self._w:
            raise MemoryError("silk_world_create failed")

    def __del__(self) -> None:
        w = getattr(self, "_w", None)
        if w:
            lib.silk_world_destroy(w)
            self._w = None

    # --- global ---
    def init(self, backend: Backend = Backend.GPU) -> Result:
        return _result(lib.silk_world_init(self._w, int(backend)), self._w)

    def set_global_config(self, config: GlobalConfig) -> Result:
        c = config.to_c()
        return _result(lib.silk_set_global_config(self._w, C.byref(c)), self._w)

    def clear(self) -> None:
        lib.silk_clear(self._w)

    # --- solver ---
    def solver_step(self) -> Result:
        return _result(lib.silk_solver_step(self._w), self._w)

    def solver_reset(self) -> Result:
        return _result(lib.silk_solver_reset(self._w), self._w)

    # --- cloth ---
    def add_cloth(self, cloth_config: ClothConfig, collision_config: CollisionConfig,
                  verts, faces, pin_index=()) -> tuple[Result, int]:
        v, f, p = _f32(verts), _i32(faces), _i32(pin_index)
        h = C.c_uint32(0)
        cc, col = cloth_config.to_c(), collision_config.to_c()
        st = lib.silk_add_cloth(self._w, C.byref(cc), C.byref(col), v, v.size, f, f.size,
                                p.ctypes.data if p.size else None, p.size, C.byref(h))
        return _result(st, self._w), int(h.value)

    def remove_cloth(self, handle: int) -> Result:
        return _result(lib.silk_remove_cloth(self._w, handle), self._w)

    def get_cloth_position(self, handle: int, position: np.ndarray) -> Result:
        """Fill ``position`` (float32, size 3 * vertex count) in mesh order."""
        if position.dtype != np.float32 or not position.flags.c_contiguous:
            raise TypeError("position must be a contiguous float32 array")
        return _result(lib.silk_get_cloth_position(self._w, handle, position.reshape(-1),
                                                   position.size), self._w)

    def set_cloth_config(self, handle: int, config: ClothConfig) -> Result:
        c = config.to_c()
        return _result(lib.silk_set_cloth_config(self._w, handle, C.byref(c)), self._w)

    def set_cloth_collision_config(self, handle: int, config: CollisionConfig) -> Result:
        c = config.to_c()
        return _result(lib.silk_set_cloth_collision_config(self._w, handle, C.byref(c)),
                       self._w)

    def set_cloth_pin_index(self, handle: int, pin_index) -> Result:
        p = _i32(pin_index)
        return _result(lib.silk_set_cloth_pin_index(self._w, handle,
                                                    p.ctypes.data if p.size else None,
                                                    p.size), self._w)

    def set_cloth_pin_position(self, handle: int, position) -> Result:
        p = _f32(position)
        return _result(lib.silk_set_cloth_pin_position(self._w, handle,
                                                       p.ctypes.data if p.size else None,
                                                       p.size), self._w)

    # --- obstacle ---
    def add_obstacle(self, collision_config: CollisionConfig, verts,
                     faces) -> tuple[Result, int]:
        v, f = _f32(verts), _i32(faces)
        h = C.c_uint32(0)
        col = collision_config.to_c()
        st = lib.silk_add_obstacle(self._w, C.byref(col), v, v.size,
                                   f.ctypes.data if f.size else None, f.size, C.byref(h))
        return _result(st, self._w), int(h.value)

    def remove_obstacle(self, handle: int) -> Result:
        return _result(lib.silk_remove_obstacle(self._w, handle), self._w)

    def set_obstacle_collision_config(self, handle: int, config: CollisionConfig) -> Result:
        c = config.to_c()
        return _result(lib.silk_set_obstacle_collision_config(self._w, handle, C.byref(c)),
                       self._w)

    def set_obstacle_position(self, handle: int, position) -> Result:
        p = _f32(position)
        return _result(lib.silk_set_obstacle_position(self._w, handle, p, p.size), self._w)

    # --- extensions ---
    def set_solver_options(self, options: SolverOptions) -> Result:
        o = options.to_c()
        return _result(lib.silk_set_solver_options(self._w, C.byref(o)), self._w)

    def step_stats(self) -> StepStats:
        s = _StepStatsC()
        lib.silk_get_step_stats(self._w, C.byref(s))
        return StepStats(**{n: getattr(s, n) for n in StepStats.__dataclass_fields__})

    def set_stream(self, cuda_stream: int | None) -> Result:
        return _result(lib.silk_set_stream(self._w, cuda_stream or None), self._w)

    def profile(self, reset: bool = False) -> dict:
        p = _ProfileC()
        lib.silk_get_profile(self._w, C.byref(p), int(reset))
        return {n: getattr(p, n) for n, _ in _ProfileC._fields_}

    def set_cloth_state(self, handle: int, position, velocity=None) -> Result:
        """Restart a cloth from stored positions (and velocities; None = at
        rest), mesh order."""
        x = _f32(position)
        if velocity is None:
            return _result(lib.silk_set_cloth_state(self._w, handle, x, x.size, None, 0),
                           self._w)
        v = _f32(velocity)
        return _result(lib.silk_set_cloth_state(self._w, handle, x, x.size, v.ctypes.data,
                                                v.size), self._w)

    def get_cloth_velocity(self, handle: int, velocity: np.ndarray) -> Result:
        return _result(lib.silk_get_cloth_velocity(self._w, handle, velocity.reshape(-1),
                                                   velocity.size), self._w)

    # --- inspection ---
    def cloth_partition(self, handle: int, nv: int) -> tuple[np.ndarray, np.ndarray]:
        perm = np.zeros(nv, np.int32)
        offs = np.zeros(nv + 1, np.int32)
        n = C.c_int32(0)
        st = lib.silk_debug_cloth_partition(self._w, handle, perm, nv, offs, nv + 1,
                                            C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return perm, offs[: n.value + 1].copy()

    def cloth_matrix(self, handle: int, nv: int) -> np.ndarray:
        d = np.zeros(nv * nv, np.float64)
        st = lib.silk_debug_cloth_matrix(self._w, handle, d, d.size)
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return d.reshape(nv, nv)

    def mas_fine(self, handle: int, nbank: int, nv: int) -> tuple[np.ndarray, np.ndarray]:
        """(packed FP32 fine-bank inverses, nbank x 528; ADMM diagonal, nv)
        of the last factorisation, solver order."""
        inv = np.zeros(nbank * 528, np.float32)
        diag = np.zeros(nv, np.float32)
        st = lib.silk_debug_mas_fine(self._w, handle, inv, inv.size, diag, diag.size)
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return inv.reshape(nbank, 528), diag

    def debug_refit(self, disp=None) -> None:
        if disp is None:
            st = lib.silk_debug_refit(self._w, None, 0)
        else:
            d = _f32(disp)
            st = lib.silk_debug_refit(self._w, d.ctypes.data, d.size)
        if st:
            raise RuntimeError(_result(st, self._w).to_string())

    def debug_candidates(self, cap: int = 1 << 22) -> np.ndarray:
        out = np.zeros(5 * cap, np.int32)
        n = C.c_int32(0)
        st = lib.silk_debug_candidates(self._w, out, cap, C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return out[: 5 * min(n.value, cap)].reshape(-1, 5)

    def debug_dcd(self, t: float, activation: float, cap: int = 1 << 20) -> np.ndarray:
        out = np.zeros(7 * cap, np.int32)
        n = C.c_int32(0)
        st = lib.silk_debug_dcd(self._w, t, activation, out, cap, C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return out[: 7 * min(n.value, cap)].reshape(-1, 7)

    def debug_contacts(self, cap: int = 1 << 20) -> np.ndarray:
        """Active contact keys of the last step, rows (type, obj_a, obj_b,
        i0..i3) in canonical order."""
        out = np.zeros(7 * cap, np.int32)
        n = C.c_int32(0)
        st = lib.silk_debug_contacts(self._w, out, cap, C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return out[: 7 * min(n.value, cap)].reshape(-1, 7)

    def debug_min_toi(self, time_start: float, max_time: float, min_separation: float,
                      prune: bool = False) -> tuple[float, int, int]:
        toi = C.c_float(0)
        nq, nh = C.c_int32(0), C.c_int32(0)
        st = lib.silk_debug_min_toi(self._w, time_start, max_time, min_separation,
                                    int(prune), C.byref(toi), C.byref(nq), C.byref(nh))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return toi.value, nq.value, nh.value

    def set_warm_start_model(self, params: np.ndarray | None) -> Result:
        if params is None:
            return _result(lib.silk_set_warm_start_model(self._w, None, 0), self._w)
        p = _f32(params)
        return _result(lib.silk_set_warm_start_model(self._w, p.ctypes.data, p.size), self._w)

    def warm_start_samples(self, handle: int, nv: int):
        """(features n x 16, targets n x 4) of the last step, or None."""
        f = np.zeros((nv, 16), np.float32)
        t = np.zeros((nv, 4), np.float32)
        valid = C.c_int32(0)
        st = lib.silk_get_warm_start_samples(self._w, handle, f.reshape(-1), t.reshape(-1), nv,
                                             C.byref(valid))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return (f, t) if valid.value else None

    def iterate_samples(self, cap: int = 1 << 19):
        """Iterate-model samples of the last step (capture_samples bit 2):
        (features n x 16, targets n x 4)."""
        f = np.zeros((cap, 16), np.float32)
        t = np.zeros((cap, 4), np.float32)
        n = C.c_int32(0)
        st = lib.silk_get_iterate_samples(self._w, f.reshape(-1), t.reshape(-1), cap, C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        return f[: n.value], t[: n.value]

    def debug_cg_trace(self, handle: int) -> dict | None:
        """Phase trace of the last CG solve (solver option profile = 2):
        kernel ns and cycles, the kernel form (0 streaming, 1 resident) and,
        per traced iteration, the cycles between consecutive phase stamps
        (16 slots; slot 0 is measured from the previous iteration's last)."""
        buf = np.zeros(8 + 64 * 16, np.int64)
        n = C.c_int32(0)
        st = lib.silk_debug_cg_trace(self._w, handle, buf.ctypes.data, buf.size, C.byref(n))
        if st:
            raise RuntimeError(_result(st, self._w).to_string())
        if n.value == 0:
            return None
        k = int(buf[4])
        stamps = buf[8: 8 + 16 * k].reshape(k, 16)
        phases = None
        if k > 1:
            prev = np.concatenate([[stamps[0, 0]], stamps[:-1, 15]])
            phases = np.diff(np.concatenate([prev[:, None], stamps], axis=1), axis=1)[1:]
        return {"ns": int(buf[2] - buf[0]), "cycles": int(buf[3] - buf[1]), "iters": k,
                "form": int(buf[5]), "phase_cycles": phases}


def ccd_batch(is_vertex_face: bool, x: np.ndarray, err3, min_separation,
              tolerance: float = 1e-6, max_iter: int = 4096, max_time: float = 1.0):
    """GPU Tight-Inclusion CCD over n queries (x: n x 24 floats)."""
    x = _f32(x)
    n = x.size // 24
    ms = _f32(np.broadcast_to(np.asarray(min_separation, np.float32), (n,)))
    hit = np.zeros(n, np.int32)
    toi = np.zeros(n, np.float32)
    tup = np.zeros(n, np.float32)
    st = lib.silk_ccd_batch(int(is_vertex_face), x, n, _f32(err3), ms, tolerance, max_iter,
                            max_time, hit, toi, tup)
    if st:
        raise RuntimeError(_result(st).to_string())
    return hit.astype(bool), toi, tup


def step_many(worlds, threads: int = 0) -> list[Result]:
    """Advance independent worlds by one step each, concurrently."""
    n = len(worlds)
    arr = (C.c_void_p * max(n, 1))(*[w._w for w in worlds])
    st = (C.c_int * max(n, 1))()
    lib.silk_step_many(arr, n, threads, st)
    return [_result(st[i], worlds[i]._w) for i in range(n)]


MLP_PARAMS = 9968  # SILK_MLP_PARAMS


def mlp_forward(params, features) -> np.ndarray:
    """GPU (tensor-core) model outputs, n x 3, of feature rows n x 16."""
    f = _f32(features).reshape(-1, 16)
    out = np.zeros((len(f), 3), np.float32)
    st = lib.silk_mlp_forward(_f32(params), f.reshape(-1), len(f), out.reshape(-1))
    if st:
        raise RuntimeError(_result(st).to_string())
    return out


def mlp_loss_grad(params, features, targets) -> tuple[float, np.ndarray]:
    f = _f32(features).reshape(-1, 16)
    t = _f32(targets).reshape(-1, 4)
    grad = np.zeros(MLP_PARAMS, np.float32)
    loss = C.c_double(0)
    st = lib.silk_mlp_loss_grad(_f32(params), f.reshape(-1), t.reshape(-1), len(f), grad,
                                C.byref(loss))
    if st:
        raise RuntimeError(_result(st).to_string())
    return loss.value, grad


def mlp_train(params, features, targets, steps: int, batch: int, lr: float,
              seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Adam on the GPU; returns (trained parameters, loss per step)."""
    p = _f32(params).copy()
    f = _f32(features).reshape(-1, 16)
    t = _f32(targets).reshape(-1, 4)
    hist = np.zeros(max(steps, 1), np.float32)
    st = lib.silk_mlp_train(p, f.reshape(-1), t.reshape(-1), len(f), steps, batch, lr, seed,
                            hist.ctypes.data)
    if st:
        raise RuntimeError(_result(st).to_string())
    return p, hist[:steps]


# Mirrors SILK_CCD_NOALLOC_MAX_QUERIES / SILK_CCD_NOALLOC_MAX_ITER.
CCD_NOALLOC_MAX_QUERIES = 1 << 20
CCD_NOALLOC_MAX_ITER = 4096


def ccd_batch_noalloc(is_vertex_face: bool, x_ptr: int, n: int, err3, ms_ptr: int,
                      hit_ptr: int, toi_ptr: int, tup_ptr: int | None = None,
                      tolerance: float = 1e-6, max_iter: int = 4096,
                      max_time: float = 1.0, stream: int = 0) -> tuple[Result, int]:
    """CCD batch on caller-owned device buffers (addresses on the current
    device) that allocates nothing; returns (status, spilled query count)."""
    spilled = C.c_int32(0)
    st = lib.silk_ccd_batch_noalloc(int(is_vertex_face), x_ptr, n, _f32(err3), ms_ptr,
                                    tolerance, max_iter, max_time, hit_ptr, toi_ptr,
                                    tup_ptr, stream or None, C.byref(spilled))
    return _result(st), spilled.value


def partition_mesh(verts, faces) -> tuple[np.ndarray, np.ndarray]:
    """(perm original->solver, part offsets) of the MAS vertex partition."""
    v, f = _f32(verts), _i32(faces)
    nv = v.size // 3
    perm = np.zeros(nv, np.int32)
    offs = np.zeros(nv + 1, np.int32)
    n = C.c_int32(0)
    st = lib.silk_partition_mesh(v, v.size, f, f.size, perm, offs, offs.size, C.byref(n))
    if st:
        raise RuntimeError(_result(st).to_string())
    return perm, offs[: n.value + 1].copy()


def schedule_bank_rows(rows, width: int, slot0: int) -> tuple[np.ndarray, np.ndarray]:
    """Entry order of one bank's 32 rows (lists of (column, value bits)) in
    the resident CG's ELL slice: (columns, values), each width x 32, round j
    of row l at [j, l]."""
    assert len(rows) == 32
    ptr = np.zeros(33, np.int32)
    ptr[1:] = np.cumsum([len(r) for r in rows])
    cols = np.array([c for r in rows for c, _ in r] or [0], np.int32)
    vals = np.array([v for r in rows for _, v in r] or [0], np.int32)
    oc = np.zeros(width * 32, np.int32)
    ov = np.zeros(width * 32, np.int32)
    st = lib.silk_schedule_bank_rows(ptr, cols, vals, width, slot0, oc, ov)
    if st:
        raise RuntimeError(_result(st).to_string())
    return oc.reshape(width, 32), ov.reshape(width, 32)


def assemble_cloth_host(cloth: ClothConfig, verts, faces, dt: float):
    """Host assembly in solver order: (L dense, mass, contact weight, bending rhs)."""
    v, f = _f32(verts), _i32(faces)
    nv = v.size // 3
    L = np.zeros(nv * nv, np.float64)
    m = np.zeros(nv, np.float64)
    w = np.zeros(nv, np.float64)
    b = np.zeros(3 * nv, np.float64)
    c = cloth.to_c()
    st = lib.silk_assemble_cloth_host(C.byref(c), v, v.size, f, f.size, dt, L.ctypes.data,
                                      m.ctypes.data, w.ctypes.data, b.ctypes.data)
    if st:
        raise RuntimeError(_result(st).to_string())
    return L.reshape(nv, nv), m, w, b


def debug_coulomb(u, normal, friction) -> np.ndarray:
    """The GPU contact Gauss-Seidel's Coulomb projection of n (u, normal,
    friction) triples (n x 3 results)."""
    u = _f32(u).reshape(-1)
    nn = _f32(normal).reshape(-1)
    mu = _f32(friction).reshape(-1)
    n = mu.size
    if u.size != 3 * n or nn.size != 3 * n:
        raise ValueError("u and normal need 3 floats per friction coefficient")
    out = np.zeros(3 * n, np.float32)
    st = lib.silk_debug_coulomb(u, nn, mu, n, out)
    if st:
        raise RuntimeError(_result(st).to_string())
    return out.reshape(n, 3)


def color_contacts(verts4: np.ndarray, prio: np.ndarray) -> tuple[np.ndarray, int]:
    v = _i32(verts4)
    p = np.ascontiguousarray(np.asarray(prio, np.uint64).ravel())
    colors = np.zeros(p.size, np.int32)
    nc = C.c_int32(0)
    st = lib.silk_color_contacts(v, p, p.size, colors, C.byref(nc))
    if st:
        raise RuntimeError(_result(st).to_string())
    return colors, nc.value
