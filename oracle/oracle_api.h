/* CPU oracle for the Silk per-step cloth hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates the reference algorithms (iiiian/silk_physics) on the
 * CPU so that the CUDA product can be checked against it.  Only the test suite,
 * __graft_entry__.smoke() and the cpu_baseline / reference leg of bench.py load
 * it.  The product library never links, includes or calls anything here.
 *
 * Parity status: pinned by the reference's own known-answer tests
 * (test/friction_contact_test.cu:10-92), by the numerical-filter constants
 * derived by test/narrowphase/derive_numerical_filter.py, and by the
 * touching-box broadphase rule of test/broadphase/main.cpp:353-380.  The
 * reference itself cannot be compiled in this environment (its dependencies
 * are fetched from the network), so whole-step trajectories are pinned only
 * through this restatement.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  float acceleration[3];
  int max_outer_iteration;
  int max_inner_iteration;
  float dt;
  float linear_solver_abs_tol;
  float linear_solver_rel_tol_min;
  float linear_solver_rel_tol_max;
  float initial_linear_rel_tol;
  float admm_abs_tol;
  float admm_rel_tol;
  /* > 0: CG relative tolerance fixed to this value (bench mode). */
  float fixed_linear_rel_tol;
  int cg_max_iter;
} oracle_global_config;

typedef struct {
  float elastic_stiffness;
  float bending_stiffness;
  float density;
  float damping;
} oracle_cloth_config;

typedef struct {
  int is_collision_on;
  int is_self_collision_on;
  int group;
  float restitution;
  float friction;
} oracle_collision_config;

typedef struct {
  int outer_iterations;
  int admm_iterations;   /* summed over outer iterations */
  int cg_iterations;     /* summed over all CG solves */
  int cg_solves;
  int contacts;
  int colors;
  int ccd_queries;
  int ccd_hits;
  float min_toi;         /* last outer iteration, in step units */
} oracle_stats;

void* oracle_world_new(int fp64);
void oracle_world_free(void* w);
int oracle_set_global_config(void* w, const oracle_global_config* c);
/* perm: original vertex -> solver vertex; part_offsets: CSR offsets of the
 * <=32-vertex partitions in solver order (defines the MAS banks). */
int oracle_add_cloth(void* w, const oracle_cloth_config* cc,
                     const oracle_collision_config* col, const float* verts,
                     int nv, const int* faces, int nf, const int* pins,
                     int npins, const int* perm, const int* part_offsets,
                     int nparts, uint32_t* handle);
int oracle_add_obstacle(void* w, const oracle_collision_config* col,
                        const float* verts, int nv, const int* faces, int nf,
                        uint32_t* handle);
int oracle_set_obstacle_position(void* w, uint32_t h, const float* pos, int n);
int oracle_set_cloth_pin_position(void* w, uint32_t h, const float* pos, int n);
int oracle_solver_step(void* w);
/* Overwrite a cloth's positions and velocities (original vertex order). */
int oracle_set_cloth_state(void* w, uint32_t h, const float* x, const float* v,
                           int n);
int oracle_get_cloth_position(void* w, uint32_t h, float* out, int n);
int oracle_get_cloth_position_f64(void* w, uint32_t h, double* out, int n);
/* Velocities (original vertex order). */
int oracle_get_cloth_velocity(void* w, uint32_t h, float* out, int n);
int oracle_get_stats(void* w, oracle_stats* s);

/* Assembled static system of one cloth, solver order: the scalar V x V matrix
 * L such that H = L (x) I3 is returned as dense row-major (small meshes). */
int oracle_cloth_dense_scalar_matrix(void* w, uint32_t h, double* out, int nv);
/* Full 3V x 3V matrix assembled the reference way (9x9 per face scatter). */
int oracle_cloth_dense_full_matrix(void* w, uint32_t h, double* out, int n);
int oracle_cloth_vectors(void* w, uint32_t h, double* mass3, double* contact_w,
                         double* bending_rhs, int n);

/* Candidate pairs of the current collider state (after the last refit):
 * out rows = (kind, obj_a, idx_a, obj_b, idx_b); kind 0 = point-triangle
 * (a = triangle, b = point), 1 = edge-edge. Returns count (may exceed cap). */
int oracle_debug_candidates(void* w, int* out, int cap);
/* Refit colliders of every cloth to (t0 = current, t1 = current + disp),
 * disp in original vertex order per cloth concatenated. */
int oracle_debug_refit(void* w, const float* disp, int n);
/* Active DCD contacts at collider time t: rows of 4 vertex ids + type + obj
 * ids (canonical key order), count returned. */
int oracle_debug_dcd(void* w, float t, float dact, int* keys, int cap);
/* Minimum time of impact over all candidates of the current refit. */
float oracle_debug_min_toi(void* w, float time_start, float max_time, float ms,
                           int* n_queries, int* n_hits);

/* Component restatements used by the known-answer tests. */
int oracle_ccd(int is_vf, const float* x24, const float* err3, float ms,
               float tol, long max_iter, int no_zero_toi, float max_time,
               float* t4, int* use_small_ms);
int oracle_exact_ee_uv(const float* x12, float eps, float* uv);
int oracle_exact_pt_uv(const float* x12, float eps, float* uv);
void oracle_solve_coulomb(const float* u3, const float* n3, float mu,
                          float* out3);
void oracle_numerical_error(const float* absmax3, int is_vf, float* out3);
/* Greedy colouring in priority order of an explicit contact graph given as a
 * list of 4 vertex ids per contact (-1 = immovable) and a priority key. */
int oracle_color_contacts(const int* verts4, const uint64_t* prio, int n,
                          int* colors);
/* 3x2 SVD clamp projection: returns vec(U clamp(S) V^T). */
void oracle_clamp_projection(const float* f6, float lo, float hi, float* out6);

#ifdef __cplusplus
}
#endif
