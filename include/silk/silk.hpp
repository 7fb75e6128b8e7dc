/// @file silk.hpp
/// @brief silk::World over the B200 C ABI (include/silk_b200.h).
///
/// Same public surface as the reference header silk/include/silk/silk.hpp
/// (lines 19-239) and silk/include/silk/result.hpp (lines 22-80): identical
/// type names, field order, defaults, method signatures, error codes and
/// "handle = 0 on failure" behaviour, so that code written against the
/// reference compiles unchanged.  Every method forwards to one extern "C"
/// function of libsilk_b200.so; no exception crosses the ABI.
///
/// Differences: World::init(Backend::CPU) returns InvalidConfig (only the
/// GPU path is provided), and silk::Result is header-only here.
#pragma once

#include <cstdint>
#include <memory>
#include <span>
#include <string>
#include <string_view>
#include <utility>

#include "../silk_b200.h"

namespace silk {

enum class ErrorCode {
  Unknown,
  NotInitialized,
  InvalidConfig,
  TooManyBody,
  InvalidHandle,
  InvalidMesh,
  InvalidPin,
  InvalidPosition,
  CholeskyDecompositionFail,
  NeedInitSolverFirst,
  IterativeSolveFail,
  NoCudaSupport
};

class Result {
 public:
  bool success = true;
  ErrorCode code = ErrorCode::Unknown;
  std::string detail;

  static Result ok() { return Result(); }
  static Result error(ErrorCode c, std::string_view d = {}) {
    Result r;
    r.success = false;
    r.code = c;
    r.detail = d;
    return r;
  }
  operator bool() const { return success; }
  std::string to_string() const {
    static const char* names[] = {"Unknown",        "NotInitialized",
                                  "InvalidConfig",  "TooManyBody",
                                  "InvalidHandle",  "InvalidMesh",
                                  "InvalidPin",     "InvalidPosition",
                                  "CholeskyDecompositionFail",
                                  "NeedInitSolverFirst",
                                  "IterativeSolveFail", "NoCudaSupport"};
    if (success) return "OK";
    std::string s = names[static_cast<int>(code)];
    if (!detail.empty()) s += ". Reason: " + detail + ".";
    return s;
  }

 private:
  Result() = default;
};

struct MeshConfig {
  std::span<const float> verts;
  std::span<const int> faces;
};

struct CollisionConfig {
  bool is_collision_on = true;
  bool is_self_collision_on = true;
  int group = 0;
  float restitution = 0.3f;
  float friction = 0.3f;
};

struct ClothConfig {
  float elastic_stiffness = 100.0f;
  float bending_stiffness = 0.0001f;
  float density = 0.1f;
  float damping = 0.01f;
};

struct GlobalConfig {
  float acceleration_x = 0.0f;
  float acceleration_y = 0.0f;
  float acceleration_z = -10.0f;
  int max_outer_iteration = 100;
  int max_inner_iteration = 100;
  float dt = 1.0f / 60.0f;
  float linear_solver_abs_tol = 1e-7f;
  float linear_solver_rel_tol_min = 1e-6f;
  float linear_solver_rel_tol_max = 1e-3f;
  float initial_linear_rel_tol = 1e-2f;
  float admm_abs_tol = 1e-5f;
  float admm_rel_tol = 1e-3f;
};

enum class Backend { CPU, GPU };

class World {
 public:
  World() : w_(silk_world_create(), &silk_world_destroy) {}
  ~World() = default;
  World(const World&) = delete;
  World(World&&) = default;
  World& operator=(const World&) = delete;
  World& operator=(World&&) = default;

  [[nodiscard]] Result init(Backend backend) {
    return wrap(silk_world_init(w_.get(), backend == Backend::GPU ? SILK_BACKEND_GPU
                                                                  : SILK_BACKEND_CPU));
  }

  [[nodiscard]] Result set_global_config(GlobalConfig c) {
    silk_global_config g{c.acceleration_x, c.acceleration_y, c.acceleration_z,
                         c.max_outer_iteration, c.max_inner_iteration, c.dt,
                         c.linear_solver_abs_tol, c.linear_solver_rel_tol_min,
                         c.linear_solver_rel_tol_max, c.initial_linear_rel_tol,
                         c.admm_abs_tol, c.admm_rel_tol};
    return wrap(silk_set_global_config(w_.get(), &g));
  }

  void clear() { silk_clear(w_.get()); }

  [[nodiscard]] Result solver_step() { return wrap(silk_solver_step(w_.get())); }
  [[nodiscard]] Result solver_reset() { return wrap(silk_solver_reset(w_.get())); }

  [[nodiscard]] Result add_cloth(ClothConfig cloth_config,
                                 CollisionConfig collision_config,
                                 MeshConfig mesh_config,
                                 std::span<const int> pin_index,
                                 uint32_t& handle) {
    silk_cloth_config cc = to_c(cloth_config);
    silk_collision_config col = to_c(collision_config);
    return wrap(silk_add_cloth(w_.get(), &cc, &col, mesh_config.verts.data(),
                               (int64_t)mesh_config.verts.size(),
                               mesh_config.faces.data(),
                               (int64_t)mesh_config.faces.size(), pin_index.data(),
                               (int64_t)pin_index.size(), &handle));
  }

  [[nodiscard]] Result remove_cloth(uint32_t handle) {
    return wrap(silk_remove_cloth(w_.get(), handle));
  }

  [[nodiscard]] Result get_cloth_position(uint32_t handle,
                                          std::span<float> position) const {
    return wrap(silk_get_cloth_position(w_.get(), handle, position.data(),
                                        (int64_t)position.size()));
  }

  [[nodiscard]] Result set_cloth_config(uint32_t handle, ClothConfig config) {
    silk_cloth_config cc = to_c(config);
    return wrap(silk_set_cloth_config(w_.get(), handle, &cc));
  }

  [[nodiscard]] Result set_cloth_collision_config(uint32_t handle,
                                                  CollisionConfig config) {
    silk_collision_config c = to_c(config);
    return wrap(silk_set_cloth_collision_config(w_.get(), handle, &c));
  }

  [[nodiscard]] Result set_cloth_pin_index(uint32_t handle,
                                           std::span<const int> pin_index) {
    return wrap(silk_set_cloth_pin_index(w_.get(), handle, pin_index.data(),
                                         (int64_t)pin_index.size()));
  }

  [[nodiscard]] Result set_cloth_pin_position(uint32_t handle,
                                              std::span<const float> position) {
    return wrap(silk_set_cloth_pin_position(w_.get(), handle, position.data(),
                                            (int64_t)position.size()));
  }

  [[nodiscard]] Result add_obstacle(CollisionConfig collision_config,
                                    MeshConfig mesh_config, uint32_t& handle) {
    silk_collision_config col = to_c(collision_config);
    return wrap(silk_add_obstacle(w_.get(), &col, mesh_config.verts.data(),
                                  (int64_t)mesh_config.verts.size(),
                                  mesh_config.faces.data(),
                                  (int64_t)mesh_config.faces.size(), &handle));
  }

  [[nodiscard]] Result remove_obstacle(uint32_t handle) {
    return wrap(silk_remove_obstacle(w_.get(), handle));
  }

  [[nodiscard]] Result set_obstacle_collision_config(uint32_t handle,
                                                     CollisionConfig config) {
    silk_collision_config c = to_c(config);
    return wrap(silk_set_obstacle_collision_config(w_.get(), handle, &c));
  }

  [[nodiscard]] Result set_obstacle_position(uint32_t handle,
                                             std::span<const float> position) {
    return wrap(silk_set_obstacle_position(w_.get(), handle, position.data(),
                                           (int64_t)position.size()));
  }

 private:
  std::unique_ptr<silk_world, void (*)(silk_world*)> w_;

  Result wrap(silk_status s) const {
    if (s == SILK_OK) return Result::ok();
    return Result::error(static_cast<ErrorCode>(s - 1),
                         silk_world_last_error(w_.get()));
  }
  static silk_cloth_config to_c(const ClothConfig& c) {
    return {c.elastic_stiffness, c.bending_stiffness, c.density, c.damping};
  }
  static silk_collision_config to_c(const CollisionConfig& c) {
    return {c.is_collision_on ? 1 : 0, c.is_self_collision_on ? 1 : 0, c.group,
            c.restitution, c.friction};
  }
};

}  // namespace silk
