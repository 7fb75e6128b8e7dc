// World: host orchestration of the per-step cloth pipeline on one GPU.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/silk_b200.h"
#include "common.cuh"
#include "host_setup.hpp"
#include "mas_cg.cuh"
#include "solver_kernels.cuh"

namespace silkb {

// Owning device allocation.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), cap(o.cap) {
    o.p = nullptr;
    o.n = o.cap = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      cap = o.cap;
      o.p = nullptr;
      o.n = o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  // Size the buffer to `count` elements.  The storage only grows: a smaller
  // or equal request reuses it (cudaFree synchronises the whole device, and
  // the per-outer-iteration buffers of the contact build are resized often).
  // Contents are unspecified afterwards.  All work of a world is ordered on
  // its stream, so reusing storage that earlier launches read is safe.
  void alloc(size_t count) {
    if (count <= cap && p) {
      n = count;
      return;
    }
    // A growing size (the contact build's buffers follow the contact count
    // from call to call) takes at least half the capacity more each time, so
    // it reallocates a logarithmic number of times.
    const size_t grown = cap + cap / 2;
    const size_t c = count > grown ? count : grown;
    reset();
    cap = c;
    n = count;
    if (c) CUDA_CHECK(cudaMalloc(&p, c * sizeof(T)));
  }
  void zero(cudaStream_t st) {
    if (n) CUDA_CHECK(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  }
  void upload(const std::vector<T>& h, cudaStream_t st) {
    alloc(h.size());
    if (n) CUDA_CHECK(cudaMemcpyAsync(p, h.data(), n * sizeof(T),
                                      cudaMemcpyHostToDevice, st));
  }
};

struct ClothDev {
  DevBuf<int> sl_ptr, sl_w;
  DevBuf<int2> ent;
  DevBuf<float> Ldiag;
  DevBuf<double> Lvals;
  DevBuf<int> part_off;
  DevBuf<int4> cmap;
  struct Level {
    DevBuf<int> fill_src, cco_base, ncco;
    DevBuf<signed char> slot_cco;
    DevBuf<float> M;
    DevBuf<__nv_bfloat16> Mb;
    DevBuf<float4> zout, rout;
    DevBuf<int> member_off, member;  // levels above the first: nodes summed into each node
  };
  Level fine;
  std::vector<Level> coarse;
  struct Gal {
    DevBuf<int> src_off, src, diag_off, diag;
    DevBuf<double> vals;
  };
  std::vector<Gal> gal;
  DevBuf<float4> r, z0, p, Ap;
  DevBuf<double> partials, coarse_partial;
  DevBuf<unsigned> barrier;
  DevBuf<int> result;
  DevBuf<float> result_rr;
  DevBuf<int> stats;  // accumulated [iterations, solves] of this cloth
  DevBuf<long long> cg_trace;  // phase trace of the last CG solve (profile >= 2)
  DevBuf<int> rb_ptr, rb_w;   // resident form: ELL slices per fine bank
  DevBuf<int2> rent;
  DevBuf<int> res_halo_off, res_halo_col;  // resident form: per-block halo vertices
  bool res_halo_full = false;              // every off-block column is in a halo
  int res_blocks = 0;         // resident form: blocks (0 = streaming form only)
  int res_grid = 0;           // cg_resident_grid(res_blocks)
  int dsm_ctas = 0;           // cluster form with redundant coarse levels: CTAs (0 = not used)
  int dsm_f = 0;              // its fine banks per CTA
  int tm_cols = 0, tm_rw = 0;  // cluster / resident rows in tensor memory (CgArgs::tm_cols / tm_rw)
  DevBuf<int> dsm_push_off, dsm_push;  // its pushes of fine-level z to other CTAs' halos
  CgArgs cg;
  int cg_grid = 1;
  double bytes_per_iter_fp32 = 0.0;  // algorithmic DRAM bytes per CG iteration
  double bytes_per_iter_bf16 = 0.0;
};

struct Cloth {
  uint32_t handle = 0;
  silk_cloth_config cfg{};
  silk_collision_config coll{};
  std::vector<float> rest;   // original order, 3 per vertex
  std::vector<int> faces;    // original ids
  std::vector<int> pins;     // original ids
  std::vector<float> pin_pos;
  std::vector<float> x_host, v_host;  // original order; valid if !on_device
  bool on_device = false;
  std::unique_ptr<ClothSetup> setup;
  bool setup_valid = false;
  ClothDev dev;
  int voff = 0, foff = 0, eoff = 0;
  int nv() const { return (int)rest.size() / 3; }
  int nf() const { return (int)faces.size() / 3; }
};

struct Obstacle {
  uint32_t handle = 0;
  silk_collision_config coll{};
  std::vector<float> cur, prev;  // 3 per vertex
  std::vector<int> faces;
  bool is_static = true, is_static_twice = true;
  bool positions_dirty = true;
  int nv() const { return (int)cur.size() / 3; }
  int nf() const { return (int)faces.size() / 3; }
};

class CollisionSystem;

class World {
 public:
  World();
  ~World();

  std::string last_error;
  bool initialized = false;
  int device = 0;  // CUDA device the world was initialised on

  silk_status init(int backend);
  silk_status set_global_config(const silk_global_config& c);
  void clear();
  silk_status solver_step();
  silk_status solver_reset();
  silk_status add_cloth(const silk_cloth_config& cc,
                        const silk_collision_config& col, const float* v,
                        int64_t nvf, const int* f, int64_t nfi, const int* pins,
                        int64_t npins, uint32_t* handle);
  silk_status remove_cloth(uint32_t h);
  silk_status get_cloth_position(uint32_t h, float* out, int64_t n);
  silk_status set_cloth_config(uint32_t h, const silk_cloth_config& c);
  silk_status set_cloth_collision_config(uint32_t h,
                                         const silk_collision_config& c);
  silk_status set_cloth_pin_index(uint32_t h, const int* pins, int64_t n);
  silk_status set_cloth_pin_position(uint32_t h, const float* pos, int64_t n);
  silk_status add_obstacle(const silk_collision_config& col, const float* v,
                           int64_t nvf, const int* f, int64_t nfi,
                           uint32_t* handle);
  silk_status remove_obstacle(uint32_t h);
  silk_status set_obstacle_collision_config(uint32_t h,
                                            const silk_collision_config& c);
  silk_status set_obstacle_position(uint32_t h, const float* pos, int64_t n);
  silk_status set_solver_options(const silk_solver_options& o);
  silk_status set_stream(void* s);
  silk_status get_profile(silk_profile* p, bool reset);
  silk_status debug_cg_trace(uint32_t h, int64_t* out, int64_t cap, int32_t* n);
  silk_status get_cloth_velocity(uint32_t h, float* out, int64_t n);
  silk_status set_cloth_state(uint32_t h, const float* x, int64_t nx, const float* v,
                              int64_t nvel);
  silk_status set_warm_start_model(const float* params, int64_t n);
  silk_status get_warm_start_samples(uint32_t h, float* feat, float* target, int64_t nv,
                                     int* valid);
  silk_status get_iterate_samples(float* feat, float* target, int64_t cap, int* n);

  // Inspection.
  silk_status debug_partition(uint32_t h, int* perm, int64_t perm_len,
                              int* offs, int64_t cap, int* nparts);
  silk_status debug_matrix(uint32_t h, double* dense, int64_t n);
  silk_status debug_mas_fine(uint32_t h, float* inv, int64_t ninv, float* diag, int64_t ndiag);
  silk_status debug_refit(const float* disp, int64_t n);
  silk_status debug_candidates(int* out, int64_t cap, int* n);
  silk_status debug_dcd(float t, float dact, int* keys, int64_t cap, int* n);
  silk_status debug_contacts(int* keys, int64_t cap, int* n);
  silk_status debug_min_toi(float ts, float mt, float ms, bool prune, float* toi,
                            int* nq, int* nh);

  silk_step_stats stats{};

  // ---- state shared with the collision system ----
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  silk_global_config g{};
  silk_solver_options opt{};
  std::vector<std::unique_ptr<Cloth>> cloths;
  std::vector<std::unique_ptr<Obstacle>> obstacles;
  int nv_total = 0, nf_total = 0;
  // Global per-vertex arrays (solver order, cloths concatenated).
  DevBuf<float4> sx, sv, prev_v, outer, outer_v, x;
  DevBuf<float> mass, damp, lhs, contact_w, contact_w_base;
  DevBuf<float4> bending_rhs, rhs, inertia, pin_target, pin_lambda;
  DevBuf<float4> contact_p, contact_p_prev, contact_eta;
  DevBuf<unsigned char> pin_flag;
  DevBuf<int4> faces_d;
  DevBuf<float4> B0, B1, zu, zold;
  DevBuf<int> vf_off, vf_list;
  DevBuf<double> face_partials, vertex_partials;
  DevBuf<AdmmControl> ctl;
  AdmmControl ctl_host_{};          // last control block read by admm_solve
  const int* cg_skip_ = nullptr;    // AdmmControl::done while an ADMM solve is enqueued
  int solve_resident_ = 0, solve_cluster_ = 0;  // CG launches of the solve, by form
  DevBuf<int> cg_fail;  // kFail* bits: a bounded device wait gave up, a bank pivot failed
  // Learned warm start: model, step history, features and training samples.
  DevBuf<float> mlp_params, mlp_out, warm_feat, warm_tgt;
  DevBuf<uint16_t> mlp_image_buf, mlp2_image_buf;  // BF16 weight images of the two models
  DevBuf<float4> hist1, hist2, step_start, ypred, xpred;
  // ADMM-extrapolated CG start: the previous ADMM iterate and 2 x_k - x_(k-1).
  DevBuf<float4> admm_prev, admm_ext;
  bool admm_ext_ready = false;
  DevBuf<int> ring_off, ring;
  // Learned iterate start: second model, the last ADMM iterates (a ring of
  // three: at iteration k, slot k % 3 receives x_(k-1) before the solve),
  // scale, features, prediction and the step's training samples.
  DevBuf<float> mlp2_params, iter_feat, iter_out, iter_sigma, iter_samp_feat, iter_samp_tgt;
  DevBuf<float4> iter_hist0, iter_hist1, iter_hist2, iter_pred;
  DevBuf<int> iter_samp_n;
  bool has_iter_model = false;
  bool iter_ready = false;  // iter_pred holds a prediction for the coming solve
  bool has_model = false;
  bool samples_valid = false;
  bool warm_first_ = false;  // the current outer iteration is the step's first
  int pinned_dof = 0;
  silk_profile prof{};
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events, events_other, events_gs;
  size_t events_used = 0, events_other_used = 0, events_gs_used = 0;
  std::pair<cudaEvent_t, cudaEvent_t>* next_event_pair(
      std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& pool, size_t& used);

  Cloth* find_cloth(uint32_t h);
  Obstacle* find_obstacle(uint32_t h);
  SolverView view();

 private:
  uint32_t next_handle_ = 1;
  bool layout_valid_ = false;
  bool pins_dirty_ = true;
  float layout_dt_ = -1.0f;
  std::unique_ptr<CollisionSystem> coll_;

  void ensure_stream();
  void invalidate_layout();
  void ensure_layout();
  void build_cloth_device(Cloth& c);
  void build_resident_layout(Cloth& c);
  void upload_pins();
  void factorize(Cloth& c, cudaStream_t st);
  void cg_solve(Cloth& c, float rel_tol, bool first, cudaStream_t st);
  void ensure_cloth_streams(size_t n);
  std::vector<cudaStream_t> cloth_streams_;  // per-cloth CG streams (multi-cloth worlds)
  std::vector<cudaEvent_t> cloth_done_;
  cudaEvent_t fork_ev_ = nullptr;
  bool warm_active() const {
    return (has_model && opt.learned_warm_start) || (opt.capture_samples & 1);
  }
  float warm_sigma() const;
  bool admm_solve();  // false on divergence
  void sync();
};

}  // namespace silkb
