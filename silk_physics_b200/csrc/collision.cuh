// Collision pipeline: colliders, OIBVH-style broadphase, DCD active contacts,
// Tight-Inclusion CCD and the coloured Gauss-Seidel contact projection.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"

namespace silkb {

class World;
struct CollisionImpl;

class CollisionSystem {
 public:
  explicit CollisionSystem(World& w);
  ~CollisionSystem();

  // Rebuild colliders after a change of the world layout.
  void rebuild();
  // Smallest bbox padding over all colliders (main_loop.cu:156-162).
  float scene_padding() const;
  bool has_colliders() const;
  // Obstacle positions for this step (obstacle_assembler.cu:50-63).
  void refresh_obstacles();
  // Cloth collider trajectories t0 -> t1 (global solver-order states).
  void refit(const float4* cloth_t1, const float4* cloth_t0);
  // New step: empty contact set (contact_constraints.cu:413-434).
  void begin_step();
  // DCD at collider time t; appends new contacts.  Returns the number added.
  int append_active(float time, float activation);
  // Earliest time of impact over [time_start, time_start + max_time].  With
  // prune, searches that cannot lower the minimum stop early (same minimum;
  // n_hits then counts completed searches only).
  float min_toi(float time_start, float max_time, float min_separation,
                int* n_queries, int* n_hits, bool prune = true);
  // Contact projection of one ADMM iteration (after contact_init); with
  // skip set (AdmmControl::done of the running ADMM solve) the kernels return
  // at entry once the solve has ended.
  void contact_solve(const int* skip = nullptr) {
    gs_skip_ = skip;
    contact_solve_launch();
  }
  int contact_count() const;
  int color_count() const;
  const int* active_dof_device() const;
  int last_candidates() const;
  double last_gather_ms = 0.0;  // host wall time of the last candidate gathering
  // Narrowphase of the last min_toi (CUDA events): first and second pass,
  // queries that ran the second pass.
  double last_first_pass_ms = 0.0, last_second_pass_ms = 0.0;
  int last_second_pass_queries = 0;
  // Host wall time of the parts of the last append_active: candidate
  // gathering, contact build (DCD kernel, dedup, records, incidence),
  // colouring and the Gauss-Seidel layout.
  double last_dcd_gather_ms = 0.0, last_dcd_build_ms = 0.0, last_dcd_color_ms = 0.0,
         last_dcd_layout_ms = 0.0;

  // Inspection.
  int debug_candidates(int* out, int64_t cap);
  int debug_dcd(float t, float dact, int* keys, int64_t cap);
  // Active contact set of the last step (keys in canonical order).
  int debug_contacts(int* keys, int64_t cap);

 private:
  void contact_solve_launch();
  const int* gs_skip_ = nullptr;
  World& w_;
  std::unique_ptr<CollisionImpl> impl_;
};

// Standalone operators.
void ccd_batch_host(bool vf, const float* x, int64_t n, const float* err3,
                    const float* ms, float tol, int max_iter, float max_time,
                    int* hit, float* toi, float* t_upper);
int color_contacts_host(const int* verts4, const uint64_t* prio, int64_t n,
                        int* colors);
// The contact Gauss-Seidel's Coulomb projection (coulomb_project) on n
// (free displacement, unit normal, friction) triples.
void coulomb_debug_host(const float* u, const float* nrm, const float* mu, int64_t n,
                        float* out);

// CCD batch on caller-owned device buffers of the current device that
// allocates no memory: all working memory is a static device array.
constexpr int kNoAllocMaxQueries = 1 << 20;
constexpr int kNoAllocMaxIter = 4096;
constexpr int kNoAllocSpillSlots = 64;
enum class NoAllocStatus { kOk, kBadArgument, kBeyondLimits, kCudaError, kStorageExhausted };
NoAllocStatus ccd_batch_noalloc(bool vf, const float* x, int64_t n, const float* err3,
                                const float* ms, float tol, int max_iter, float max_time,
                                int* hit, float* toi, float* t_upper, cudaStream_t stream,
                                int* n_spilled);

}  // namespace silkb
