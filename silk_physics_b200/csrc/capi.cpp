// extern "C" boundary: every entry point of include/silk_b200.h.  Exceptions
// never cross the ABI; they become SILK_ERR_UNKNOWN with a detail string.
#include <atomic>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "../../include/silk_b200.h"
#include "collision.cuh"
#include "learned.cuh"
#include "world.hpp"

using silkb::World;

struct silk_world {
  World impl;
};

namespace {

template <class F>
silk_status guard(silk_world* w, F&& f) {
  if (!w) return SILK_ERR_INVALID_CONFIG;
  try {
    return f(w->impl);
  } catch (const std::exception& e) {
    w->impl.last_error = e.what();
    return SILK_ERR_UNKNOWN;
  }
}

template <class F>
silk_status guard_init(silk_world* w, F&& f) {
  if (!w) return SILK_ERR_INVALID_CONFIG;
  if (!w->impl.initialized) return SILK_ERR_NOT_INITIALIZED;
  return guard(w, f);
}

}  // namespace

extern "C" {

silk_world* silk_world_create(void) {
  try {
    return new silk_world();
  } catch (...) {
    return nullptr;
  }
}

void silk_world_destroy(silk_world* w) { delete w; }

const char* silk_world_last_error(const silk_world* w) {
  return w ? w->impl.last_error.c_str() : "";
}

void silk_global_config_default(silk_global_config* c) {
  c->acceleration_x = 0.0f;
  c->acceleration_y = 0.0f;
  c->acceleration_z = -10.0f;
  c->max_outer_iteration = 100;
  c->max_inner_iteration = 100;
  c->dt = 1.0f / 60.0f;
  c->linear_solver_abs_tol = 1e-7f;
  c->linear_solver_rel_tol_min = 1e-6f;
  c->linear_solver_rel_tol_max = 1e-3f;
  c->initial_linear_rel_tol = 1e-2f;
  c->admm_abs_tol = 1e-5f;
  c->admm_rel_tol = 1e-3f;
}

void silk_solver_options_default(silk_solver_options* o) {
  std::memset(o, 0, sizeof(*o));
  o->fixed_linear_rel_tol = 0.0f;
  o->cg_max_iter = 1000;
  o->mas_bf16 = 0;
}

silk_status silk_world_init(silk_world* w, int32_t backend) {
  return guard(w, [&](World& W) { return W.init(backend); });
}

silk_status silk_set_global_config(silk_world* w, const silk_global_config* c) {
  if (!c) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) { return W.set_global_config(*c); });
}

void silk_clear(silk_world* w) {
  if (w) w->impl.clear();
}

silk_status silk_solver_step(silk_world* w) {
  return guard_init(w, [&](World& W) { return W.solver_step(); });
}

silk_status silk_step_many(silk_world* const* worlds, int32_t n, int32_t threads,
                           silk_status* status) {
  if (n < 0 || (n > 0 && (!worlds || !status))) return SILK_ERR_INVALID_CONFIG;
  for (int32_t i = 0; i < n; ++i) {
    if (!worlds[i]) return SILK_ERR_INVALID_CONFIG;
    for (int32_t j = 0; j < i; ++j)
      if (worlds[j] == worlds[i]) return SILK_ERR_INVALID_CONFIG;
  }
  int hw = (int)std::thread::hardware_concurrency();
  int nt = threads > 0 ? threads : (hw > 0 ? hw : 1);
  if (nt > n) nt = n;
  std::atomic<int32_t> next{0};
  auto work = [&]() {
    for (;;) {
      int32_t i = next.fetch_add(1);
      if (i >= n) return;
      silk_world* w = worlds[i];
      if (w->impl.initialized) cudaSetDevice(w->impl.device);
      status[i] = silk_solver_step(w);
    }
  };
  std::vector<std::thread> pool;
  try {
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  } catch (...) {
    // Fewer threads than asked: the remaining ones (and this one) do the work.
  }
  work();
  for (auto& t : pool) t.join();
  for (int32_t i = 0; i < n; ++i)
    if (status[i] != SILK_OK) return status[i];
  return SILK_OK;
}

silk_status silk_solver_reset(silk_world* w) {
  return guard_init(w, [&](World& W) { return W.solver_reset(); });
}

silk_status silk_add_cloth(silk_world* w, const silk_cloth_config* cloth,
                           const silk_collision_config* collision,
                           const float* verts, int64_t verts_len,
                           const int32_t* faces, int64_t faces_len,
                           const int32_t* pins, int64_t pins_len,
                           uint32_t* handle) {
  if (handle) *handle = 0;
  if (!cloth || !collision || !handle) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) {
    return W.add_cloth(*cloth, *collision, verts, verts_len, faces, faces_len,
                       pins, pins_len, handle);
  });
}

silk_status silk_remove_cloth(silk_world* w, uint32_t handle) {
  return guard_init(w, [&](World& W) { return W.remove_cloth(handle); });
}

silk_status silk_get_cloth_position(const silk_world* w, uint32_t handle,
                                    float* position, int64_t position_len) {
  silk_world* mw = const_cast<silk_world*>(w);
  if (!position && position_len != 0) return SILK_ERR_INVALID_POSITION;
  return guard_init(mw, [&](World& W) {
    return W.get_cloth_position(handle, position, position_len);
  });
}

silk_status silk_set_cloth_config(silk_world* w, uint32_t handle,
                                  const silk_cloth_config* config) {
  if (!config) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) { return W.set_cloth_config(handle, *config); });
}

silk_status silk_set_cloth_collision_config(silk_world* w, uint32_t handle,
                                            const silk_collision_config* c) {
  if (!c) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) {
    return W.set_cloth_collision_config(handle, *c);
  });
}

silk_status silk_set_cloth_pin_index(silk_world* w, uint32_t handle,
                                     const int32_t* pins, int64_t pins_len) {
  if (!pins && pins_len != 0) return SILK_ERR_INVALID_PIN;
  return guard_init(w, [&](World& W) {
    return W.set_cloth_pin_index(handle, pins, pins_len);
  });
}

silk_status silk_set_cloth_pin_position(silk_world* w, uint32_t handle,
                                        const float* position,
                                        int64_t position_len) {
  if (!position && position_len != 0) return SILK_ERR_INVALID_PIN;
  return guard_init(w, [&](World& W) {
    return W.set_cloth_pin_position(handle, position, position_len);
  });
}

silk_status silk_add_obstacle(silk_world* w,
                              const silk_collision_config* collision,
                              const float* verts, int64_t verts_len,
                              const int32_t* faces, int64_t faces_len,
                              uint32_t* handle) {
  if (handle) *handle = 0;
  if (!collision || !handle) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) {
    return W.add_obstacle(*collision, verts, verts_len, faces, faces_len, handle);
  });
}

silk_status silk_remove_obstacle(silk_world* w, uint32_t handle) {
  return guard_init(w, [&](World& W) { return W.remove_obstacle(handle); });
}

silk_status silk_set_obstacle_collision_config(silk_world* w, uint32_t handle,
                                               const silk_collision_config* c) {
  if (!c) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) {
    return W.set_obstacle_collision_config(handle, *c);
  });
}

silk_status silk_set_obstacle_position(silk_world* w, uint32_t handle,
                                       const float* position,
                                       int64_t position_len) {
  if (!position && position_len != 0) return SILK_ERR_INVALID_POSITION;
  return guard_init(w, [&](World& W) {
    return W.set_obstacle_position(handle, position, position_len);
  });
}

silk_status silk_set_solver_options(silk_world* w, const silk_solver_options* o) {
  if (!o) return SILK_ERR_INVALID_CONFIG;
  return guard(w, [&](World& W) { return W.set_solver_options(*o); });
}

silk_status silk_get_step_stats(const silk_world* w, silk_step_stats* s) {
  if (!w || !s) return SILK_ERR_INVALID_CONFIG;
  *s = w->impl.stats;
  return SILK_OK;
}

silk_status silk_set_stream(silk_world* w, void* cuda_stream) {
  return guard_init(w, [&](World& W) { return W.set_stream(cuda_stream); });
}

silk_status silk_get_profile(silk_world* w, silk_profile* p, int32_t reset) {
  if (!p) return SILK_ERR_INVALID_CONFIG;
  return guard(w, [&](World& W) { return W.get_profile(p, reset != 0); });
}

silk_status silk_set_cloth_state(silk_world* w, uint32_t handle, const float* position,
                                 int64_t position_len, const float* velocity,
                                 int64_t velocity_len) {
  return guard_init(w, [&](World& x) {
    return x.set_cloth_state(handle, position, position_len, velocity, velocity_len);
  });
}

silk_status silk_get_cloth_velocity(const silk_world* w, uint32_t handle,
                                    float* velocity, int64_t velocity_len) {
  if (!velocity && velocity_len != 0) return SILK_ERR_INVALID_POSITION;
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.get_cloth_velocity(handle, velocity, velocity_len);
  });
}

silk_status silk_debug_cloth_partition(const silk_world* w, uint32_t handle,
                                       int32_t* perm, int64_t perm_len,
                                       int32_t* part_offsets,
                                       int64_t offsets_cap, int32_t* nparts) {
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.debug_partition(handle, perm, perm_len, part_offsets, offsets_cap,
                             nparts);
  });
}

silk_status silk_debug_cg_trace(const silk_world* w, uint32_t handle, int64_t* trace,
                               int64_t cap, int32_t* n) {
  if (!trace || !n) return SILK_ERR_INVALID_CONFIG;
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.debug_cg_trace(handle, trace, cap, n);
  });
}

silk_status silk_debug_cloth_matrix(const silk_world* w, uint32_t handle,
                                    double* dense, int64_t n_len) {
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.debug_matrix(handle, dense, n_len);
  });
}

silk_status silk_debug_mas_fine(const silk_world* w, uint32_t handle, float* inverses,
                                int64_t inverses_len, float* diag, int64_t diag_len) {
  if (!inverses || !diag) return SILK_ERR_INVALID_CONFIG;
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.debug_mas_fine(handle, inverses, inverses_len, diag, diag_len);
  });
}

silk_status silk_debug_refit(silk_world* w, const float* disp, int64_t len) {
  return guard_init(w, [&](World& W) { return W.debug_refit(disp, len); });
}

silk_status silk_debug_candidates(silk_world* w, int32_t* out, int64_t cap,
                                  int32_t* n) {
  return guard_init(w, [&](World& W) { return W.debug_candidates(out, cap, n); });
}

silk_status silk_debug_dcd(silk_world* w, float t, float activation,
                           int32_t* keys, int64_t cap, int32_t* n) {
  return guard_init(w, [&](World& W) {
    return W.debug_dcd(t, activation, keys, cap, n);
  });
}

silk_status silk_debug_contacts(silk_world* w, int32_t* keys, int64_t cap, int32_t* n) {
  if (!n || (cap > 0 && !keys)) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) { return W.debug_contacts(keys, cap, n); });
}

silk_status silk_debug_min_toi(silk_world* w, float time_start, float max_time,
                               float min_separation, int32_t prune, float* toi,
                               int32_t* n_queries, int32_t* n_hits) {
  return guard_init(w, [&](World& W) {
    return W.debug_min_toi(time_start, max_time, min_separation, prune != 0, toi,
                           n_queries, n_hits);
  });
}

silk_status silk_schedule_bank_rows(const int32_t* row_ptr, const int32_t* cols,
                                    const int32_t* vals, int32_t width, int32_t slot0,
                                    int32_t* out_cols, int32_t* out_vals) {
  if (!row_ptr || !out_cols || !out_vals || width < 0 || slot0 < 0)
    return SILK_ERR_INVALID_CONFIG;
  try {
    std::vector<std::vector<std::pair<int, int>>> rows(32);
    for (int l = 0; l < 32; ++l) {
      const int n = row_ptr[l + 1] - row_ptr[l];
      if (n < 0 || n > width || (n > 0 && (!cols || !vals))) return SILK_ERR_INVALID_CONFIG;
      for (int i = row_ptr[l]; i < row_ptr[l + 1]; ++i) rows[l].emplace_back(cols[i], vals[i]);
    }
    std::vector<std::pair<int, int>> out((size_t)width * 32);
    silkb::schedule_bank_rows(rows, width, slot0, out.data());
    for (size_t i = 0; i < out.size(); ++i) {
      out_cols[i] = out[i].first;
      out_vals[i] = out[i].second;
    }
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_partition_mesh(const float* verts, int64_t verts_len,
                                const int32_t* faces, int64_t faces_len,
                                int32_t* perm, int32_t* part_offsets,
                                int64_t offsets_cap, int32_t* nparts) {
  if (!verts || !faces || !perm || !part_offsets || !nparts || verts_len < 0 || faces_len < 0)
    return SILK_ERR_INVALID_CONFIG;
  if (!silkb::check_mesh_indices(verts, (long)verts_len, faces, (long)faces_len).empty())
    return SILK_ERR_INVALID_MESH;
  try {
    std::vector<int> p, off;
    int nv = (int)(verts_len / 3), nf = (int)(faces_len / 3);
    silkb::partition_mesh(verts, nv, faces, nf, p, off);
    *nparts = (int)off.size() - 1;
    if ((int64_t)off.size() > offsets_cap) return SILK_ERR_INVALID_CONFIG;
    std::memcpy(perm, p.data(), sizeof(int) * nv);
    std::memcpy(part_offsets, off.data(), sizeof(int) * off.size());
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_assemble_cloth_host(const silk_cloth_config* cloth,
                                     const float* verts, int64_t verts_len,
                                     const int32_t* faces, int64_t faces_len,
                                     float dt, double* dense_L, double* mass,
                                     double* contact_weight,
                                     double* bending_rhs) {
  if (!cloth || !verts || !faces) return SILK_ERR_INVALID_CONFIG;
  try {
    std::string why = silkb::check_cloth_mesh(verts, verts_len, faces, faces_len);
    if (!why.empty()) return SILK_ERR_INVALID_MESH;
    silkb::ClothParams prm;
    prm.elastic_stiffness = cloth->elastic_stiffness;
    prm.bending_stiffness = cloth->bending_stiffness;
    prm.density = cloth->density;
    prm.damping = cloth->damping;
    silkb::ClothSetup S;
    silkb::build_cloth_setup(verts, (int)(verts_len / 3), faces,
                             (int)(faces_len / 3), prm, S);
    int nv = S.nv;
    if (dense_L) {
      std::memset(dense_L, 0, sizeof(double) * (size_t)nv * nv);
      for (int i = 0; i < nv; ++i)
        for (int k = S.Lrows[i]; k < S.Lrows[i + 1]; ++k)
          dense_L[(size_t)i * nv + S.Lcols[k]] = S.Lvals[k];
    }
    if (mass)
      for (int i = 0; i < nv; ++i) mass[i] = S.mass[i];
    if (contact_weight) {
      std::vector<double> w;
      silkb::contact_weights(S, dt, w);
      for (int i = 0; i < nv; ++i) contact_weight[i] = w[i];
    }
    if (bending_rhs)
      for (int i = 0; i < 3 * nv; ++i) bending_rhs[i] = S.bending_rhs[i];
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_ccd_batch(int32_t is_vertex_face, const float* x, int64_t n,
                           const float* err3, const float* min_separation,
                           float tolerance, int32_t max_iter, float max_time,
                           int32_t* hit, float* toi, float* t_upper) {
  if (n < 0 || (n > 0 && (!x || !err3 || !min_separation || !hit || !toi)))
    return SILK_ERR_INVALID_CONFIG;
  try {
    silkb::ccd_batch_host(is_vertex_face != 0, x, n, err3, min_separation,
                          tolerance, max_iter, max_time, hit, toi, t_upper);
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_debug_coulomb(const float* u, const float* normal, const float* friction,
                              int64_t n, float* out) {
  if (n < 0 || (n > 0 && (!u || !normal || !friction || !out))) return SILK_ERR_INVALID_CONFIG;
  try {
    silkb::coulomb_debug_host(u, normal, friction, n, out);
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_color_contacts(const int32_t* verts4, const uint64_t* prio,
                                int64_t n, int32_t* colors, int32_t* ncolors) {
  if (n < 0 || (n > 0 && (!verts4 || !prio || !colors)) || !ncolors)
    return SILK_ERR_INVALID_CONFIG;
  try {
    *ncolors = silkb::color_contacts_host(verts4, prio, n, colors);
    return *ncolors >= 0 ? SILK_OK : SILK_ERR_UNKNOWN;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

static_assert(SILK_MLP_PARAMS == silkb::kMlpParams, "MLP parameter count");

silk_status silk_set_warm_start_model(silk_world* w, const float* params, int64_t n) {
  return guard_init(w, [&](World& W) { return W.set_warm_start_model(params, n); });
}

silk_status silk_get_warm_start_samples(const silk_world* w, uint32_t handle,
                                        float* features, float* targets,
                                        int64_t nverts, int32_t* valid) {
  if (!features || !targets || !valid) return SILK_ERR_INVALID_CONFIG;
  return guard_init(const_cast<silk_world*>(w), [&](World& W) {
    return W.get_warm_start_samples(handle, features, targets, nverts, valid);
  });
}

silk_status silk_get_iterate_samples(silk_world* w, float* features, float* targets,
                                     int64_t cap, int32_t* n) {
  if (!n || cap < 0 || (cap > 0 && (!features || !targets))) return SILK_ERR_INVALID_CONFIG;
  return guard_init(w, [&](World& W) { return W.get_iterate_samples(features, targets, cap, n); });
}

silk_status silk_mlp_forward(const float* params, const float* features, int64_t n,
                             float* out) {
  if (!params || n < 0 || (n > 0 && (!features || !out))) return SILK_ERR_INVALID_CONFIG;
  if (n == 0) return SILK_OK;
  try {
    silkb::mlp_forward_host(params, features, n, out);
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_mlp_loss_grad(const float* params, const float* features,
                               const float* targets, int64_t n, float* grad,
                               double* loss) {
  if (!params || n <= 0 || !features || !targets || !grad || !loss)
    return SILK_ERR_INVALID_CONFIG;
  try {
    silkb::mlp_loss_grad_host(params, features, targets, n, grad, loss);
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

silk_status silk_mlp_train(float* params, const float* features, const float* targets,
                           int64_t n, int32_t steps, int32_t batch, float lr,
                           uint64_t seed, float* loss_history) {
  if (!params || n <= 0 || !features || !targets || steps < 0) return SILK_ERR_INVALID_CONFIG;
  try {
    silkb::mlp_train_host(params, features, targets, n, steps, batch, lr, seed, loss_history);
    return SILK_OK;
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
}

static_assert(SILK_CCD_NOALLOC_MAX_QUERIES == silkb::kNoAllocMaxQueries &&
                  SILK_CCD_NOALLOC_MAX_ITER == silkb::kNoAllocMaxIter,
              "header limits match the scratch layout");

silk_status silk_ccd_batch_noalloc(int32_t is_vertex_face, const float* x,
                                   int64_t n, const float* err3,
                                   const float* min_separation, float tolerance,
                                   int32_t max_iter, float max_time,
                                   int32_t* hit, float* toi, float* t_upper,
                                   void* stream, int32_t* n_spilled) {
  using S = silkb::NoAllocStatus;
  S s = S::kCudaError;
  try {
    s = silkb::ccd_batch_noalloc(is_vertex_face != 0, x, n, err3, min_separation,
                                 tolerance, max_iter, max_time, hit, toi, t_upper,
                                 static_cast<cudaStream_t>(stream), n_spilled);
  } catch (...) {
    return SILK_ERR_UNKNOWN;
  }
  switch (s) {
    case S::kOk: return SILK_OK;
    case S::kBadArgument:
    case S::kBeyondLimits: return SILK_ERR_INVALID_CONFIG;
    default: return SILK_ERR_UNKNOWN;
  }
}

}  // extern "C"
