/* C ABI of the B200 cloth hot path.
 *
 * This is the drop-in boundary for the per-step simulation path of
 * iiiian/silk_physics: each entry point replaces one method of silk::World
 * (silk/include/silk/silk.hpp:83-239, implemented by
 * silk/src/backend/cuda/cuda_backend.cu) with plain pointers and sizes.
 * Spans become (pointer, element count) pairs, handles stay opaque uint32
 * values (0 = failure), and every call returns a silk_status that maps 1:1
 * onto silk::ErrorCode (silk/include/silk/result.hpp:22-35) shifted by one
 * so that 0 means success.  Nothing here throws across the ABI.
 *
 * Calls are synchronous like the reference's (cuda_backend.cu:87-96): the
 * world's stream is synchronised before a call returns.  A world is not
 * thread-safe.
 */
#ifndef SILK_B200_H
#define SILK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct silk_world silk_world;

/* silk::ErrorCode + 1; SILK_OK == 0. */
typedef enum {
  SILK_OK = 0,
  SILK_ERR_UNKNOWN = 1,
  SILK_ERR_NOT_INITIALIZED = 2,
  SILK_ERR_INVALID_CONFIG = 3,
  SILK_ERR_TOO_MANY_BODY = 4,
  SILK_ERR_INVALID_HANDLE = 5,
  SILK_ERR_INVALID_MESH = 6,
  SILK_ERR_INVALID_PIN = 7,
  SILK_ERR_INVALID_POSITION = 8,
  SILK_ERR_CHOLESKY_DECOMPOSITION_FAIL = 9,
  SILK_ERR_NEED_INIT_SOLVER_FIRST = 10,
  SILK_ERR_ITERATIVE_SOLVE_FAIL = 11,
  SILK_ERR_NO_CUDA_SUPPORT = 12
} silk_status;

/* silk::Backend (silk.hpp:80). Only SILK_BACKEND_GPU is provided. */
typedef enum { SILK_BACKEND_CPU = 0, SILK_BACKEND_GPU = 1 } silk_backend;

/* silk::GlobalConfig (silk.hpp:47-77), same field order and defaults. */
typedef struct {
  float acceleration_x;          /* 0 */
  float acceleration_y;          /* 0 */
  float acceleration_z;          /* -10 */
  int32_t max_outer_iteration;   /* 100 */
  int32_t max_inner_iteration;   /* 100 */
  float dt;                      /* 1/60 */
  float linear_solver_abs_tol;   /* 1e-7 */
  float linear_solver_rel_tol_min; /* 1e-6 */
  float linear_solver_rel_tol_max; /* 1e-3 */
  float initial_linear_rel_tol;  /* 1e-2 */
  float admm_abs_tol;            /* 1e-5 */
  float admm_rel_tol;            /* 1e-3 */
} silk_global_config;

/* silk::ClothConfig (silk.hpp:35-45). */
typedef struct {
  float elastic_stiffness; /* 100 */
  float bending_stiffness; /* 1e-4 */
  float density;           /* 0.1 */
  float damping;           /* 0.01 */
} silk_cloth_config;

/* silk::CollisionConfig (silk.hpp:26-33); bools as int32. */
typedef struct {
  int32_t is_collision_on;      /* 1 */
  int32_t is_self_collision_on; /* 1 */
  int32_t group;                /* 0 */
  float restitution;            /* 0.3 */
  float friction;               /* 0.3 */
} silk_collision_config;

/* Solver options with no field in silk::GlobalConfig (bench and precision
 * switches).  Defaults reproduce the reference behaviour. */
typedef struct {
  float fixed_linear_rel_tol; /* > 0: CG relative tolerance fixed (1e-5 in
                                 the headline benchmark); 0: adaptive rule of
                                 admm_solver.cu:228-233 */
  int32_t cg_max_iter;        /* 1000 (mas_cg_solver.cuh:25) */
  int32_t mas_bf16;           /* 0: FP32 bank inverses; 1: BF16 storage */
  int32_t profile;            /* 1: time the CG kernel with CUDA events;
                                 2: also record the CG phase trace */
  int32_t cg_form;            /* 0: the cluster form with redundant coarse
                                 levels where the system fits one cluster of
                                 CTAs of 8 or 16 fine banks, else the resident
                                 form where it fits, else streaming;
                                 2: resident where it fits, else streaming;
                                 1: streaming always;
                                 3, 4: as 0 and 2, the cluster and resident
                                 forms reading their matrix rows from global
                                 memory in every SpMV instead of holding them
                                 in tensor memory (applies when the solver
                                 layout is built; changing it rebuilds it) */
  int32_t learned_warm_start; /* 1: offer the loaded first-solve model's
                                 prediction as the start of each outer
                                 iteration's first CG solve and, when an
                                 iterate model is loaded, its prediction of
                                 the next ADMM iterate as the start of every
                                 later CG solve (from the third of an ADMM
                                 solve on) */
  int32_t capture_samples;    /* bit 1: record first-solve training samples;
                                 bit 2: record iterate-model training samples
                                 (256 vertices per ADMM iteration) */
  int32_t contact_gs_form;    /* 0: single-block contact Gauss-Seidel where the
                                 contacts fit it, else grid; 1: grid always */
  int32_t admm_extrapolated_start; /* 1: offer 2 x_k - x_(k-1) (the last two ADMM
                                 iterates of the same ADMM solve) as the start
                                 of each later CG solve; the plain start's
                                 residual stays the stopping reference */
  int32_t resident_halo_limit; /* > 0: at most this many (and at most 1024)
                                 off-block vertices per resident-CG block are
                                 gathered into shared memory; further ones are
                                 read from global memory and p is published
                                 through the grid (applies when the solver
                                 layout is built: first step after a change of
                                 the cloths); 0: 1024 */
  int32_t barrier_spin_limit; /* > 0: polls after which a CG grid-barrier wait
                                 gives up (the step then returns
                                 SILK_ERR_ITERATIVE_SOLVE_FAIL); 0: 2^22 */
  int32_t debug_withhold_block; /* failure-detection tests: k > 0 makes block
                                 k - 1 of a cooperative-grid CG launch skip its
                                 barrier arrivals, so the other blocks' bounded
                                 waits run out; 0: off */
  int32_t admm_check_interval; /* ADMM iterations enqueued between the host's
                                 reads of the convergence state (the device
                                 decides convergence; iterations enqueued after
                                 it do nothing); 0: 4; 1: a read after every
                                 iteration */
} silk_solver_options;

/* CUDA-event timing of the persistent CG kernel over the steps since the
 * last reset (silk_solver_options.profile = 1); the struct grew by the four
 * narrowphase fields and the six DCD fields at its end, so callers compiled
 * against a shorter silk_profile must be rebuilt.  algorithmic_bytes counts
 * compulsory DRAM traffic per CG iteration: matrix entries, MAS bank
 * inverses and each vector read or written once. */
typedef struct {
  double cg_time_ms;         /* CUDA events around the CG kernel */
  int64_t cg_launches;
  int64_t cg_iterations;
  double cg_algorithmic_bytes;
  double admm_other_ms;      /* events: face/vertex/contact kernels and the
                                convergence test run by the vertex step */
  double admm_host_ms;       /* host wall time of ADMM control (syncs) */
  double ccd_host_ms;        /* host wall time of refit + CCD */
  double dcd_host_ms;        /* host wall time of DCD + contact rebuild */
  double step_host_ms;       /* host wall time of solver_step */
  double contact_gs_ms;      /* events: contact Gauss-Seidel (part of admm_other_ms) */
  double ccd_refit_host_ms;  /* part of ccd_host_ms: collider refit and tree builds */
  double ccd_candidates_host_ms; /* part of ccd_host_ms: broadphase candidate gathering */
  double ccd_first_pass_ms;  /* events: narrowphase first pass (per-thread storage) */
  double ccd_second_pass_ms; /* events: narrowphase second pass (searches that outgrew it) */
  double ccd_second_pass_queries; /* queries that ran the second pass */
  double ccd_calls;          /* narrowphase calls (one per outer iteration) */
  double dcd_refit_host_ms;  /* part of dcd_host_ms: collider refit and tree builds */
  double dcd_candidates_host_ms; /* part of dcd_host_ms: broadphase candidate gathering */
  double dcd_build_host_ms;  /* part of dcd_host_ms: DCD kernel, dedup, contact records,
                                vertex incidence */
  double dcd_coloring_host_ms; /* part of dcd_host_ms: Jones-Plassmann colouring, groups */
  double dcd_layout_host_ms; /* part of dcd_host_ms: Gauss-Seidel slots and records */
  double dcd_calls;          /* DCD calls (step start and each rollback) */
} silk_profile;

/* Statistics of the last solver_step. */
typedef struct {
  int32_t outer_iterations;
  int32_t admm_iterations;
  int32_t cg_iterations;
  int32_t cg_solves;
  int32_t contacts;
  int32_t colors;
  int32_t ccd_queries;
  int32_t ccd_hits;
  float min_toi;
  int32_t broadphase_candidates;
  int64_t kernel_launches;
  int32_t cg_resident_solves;  /* CG solves that ran in the resident form */
  int32_t cg_first_solve_iterations; /* iterations of each outer iteration's
                                        first CG solve, summed */
  int32_t learned_starts;      /* first solves that started from the model */
  int32_t extrapolated_starts; /* solves that started from the extrapolation */
  int32_t cg_cluster_solves;   /* of the resident solves, those in the cluster form
                                  with redundant coarse levels (CTAs of 8 or 16
                                  fine banks exchanging through distributed
                                  shared memory) */
  int32_t learned_iterate_starts; /* later CG solves of an ADMM solve that started
                                  from the iterate model's prediction */
} silk_step_stats;

/* --- World lifetime (silk.hpp:92-100) ---------------------------------- */
silk_world* silk_world_create(void);
void silk_world_destroy(silk_world* w);
/* Human-readable detail of the last error of this world ("" if none). */
const char* silk_world_last_error(const silk_world* w);

/* --- Global API (silk.hpp:106-118; world.cpp:29-56) --------------------- */
silk_status silk_world_init(silk_world* w, int32_t backend);
silk_status silk_set_global_config(silk_world* w, const silk_global_config* c);
void silk_global_config_default(silk_global_config* c);
void silk_clear(silk_world* w);

/* --- Solver API (silk.hpp:124-133) -------------------------------------- */
silk_status silk_solver_step(silk_world* w);
silk_status silk_solver_reset(silk_world* w);
/* Batched step (no reference counterpart): advance n distinct, independent
 * worlds by one step each, concurrently - each world on its own CUDA stream,
 * driven by a pool of `threads` host threads (<= 0: one per hardware thread,
 * at most n).  status[i] receives world i's result; the return value is the
 * first non-OK status, or SILK_OK.  Worlds must not be used by other threads
 * during the call. */
silk_status silk_step_many(silk_world* const* worlds, int32_t n, int32_t threads,
                           silk_status* status);

/* --- Cloth API (silk.hpp:139-204) --------------------------------------- */
silk_status silk_add_cloth(silk_world* w, const silk_cloth_config* cloth,
                           const silk_collision_config* collision,
                           const float* verts, int64_t verts_len,
                           const int32_t* faces, int64_t faces_len,
                           const int32_t* pins, int64_t pins_len,
                           uint32_t* handle);
silk_status silk_remove_cloth(silk_world* w, uint32_t handle);
silk_status silk_get_cloth_position(const silk_world* w, uint32_t handle,
                                    float* position, int64_t position_len);
silk_status silk_set_cloth_config(silk_world* w, uint32_t handle,
                                  const silk_cloth_config* config);
silk_status silk_set_cloth_collision_config(silk_world* w, uint32_t handle,
                                            const silk_collision_config* c);
silk_status silk_set_cloth_pin_index(silk_world* w, uint32_t handle,
                                     const int32_t* pins, int64_t pins_len);
silk_status silk_set_cloth_pin_position(silk_world* w, uint32_t handle,
                                        const float* position,
                                        int64_t position_len);

/* --- Obstacle API (silk.hpp:210-239) ------------------------------------ */
silk_status silk_add_obstacle(silk_world* w,
                              const silk_collision_config* collision,
                              const float* verts, int64_t verts_len,
                              const int32_t* faces, int64_t faces_len,
                              uint32_t* handle);
silk_status silk_remove_obstacle(silk_world* w, uint32_t handle);
silk_status silk_set_obstacle_collision_config(silk_world* w, uint32_t handle,
                                               const silk_collision_config* c);
silk_status silk_set_obstacle_position(silk_world* w, uint32_t handle,
                                       const float* position,
                                       int64_t position_len);

/* --- Extensions (no reference counterpart) ------------------------------ */
void silk_solver_options_default(silk_solver_options* o);
silk_status silk_set_solver_options(silk_world* w, const silk_solver_options* o);
silk_status silk_get_step_stats(const silk_world* w, silk_step_stats* s);
/* Launch all device work of this world on the given cudaStream_t (NULL =
 * the world's own stream).  Lets a caller time steps with its own events. */
silk_status silk_set_stream(silk_world* w, void* cuda_stream);
/* Kernel profile accumulated since the last reset; reset = 1 clears it. */
silk_status silk_get_profile(silk_world* w, silk_profile* p, int32_t reset);
/* Vertex velocities of a cloth in mesh order (3 * vertex count floats). */
silk_status silk_get_cloth_velocity(const silk_world* w, uint32_t handle,
                                    float* velocity, int64_t velocity_len);
/* Restart a cloth from a stored state: positions and velocities in mesh
 * order (3 * vertex count floats each; velocity NULL = at rest).  Positions
 * and velocities are the whole state carried between steps (contacts are
 * rebuilt by DCD and the ADMM variables reset when a step begins,
 * main_loop.cu:140-176), so a step from here equals the step the stored
 * simulation took next.  Non-finite values give SILK_ERR_INVALID_POSITION. */
silk_status silk_set_cloth_state(silk_world* w, uint32_t handle, const float* position,
                                 int64_t position_len, const float* velocity,
                                 int64_t velocity_len);

/* Phase trace of the last CG solve of a cloth, recorded when the solver
 * option profile is 2: [0],[1] globaltimer (ns) and clock64 at kernel entry,
 * [2],[3] at exit, [4] traced iterations k (at most 64), [5] kernel form
 * (0 streaming, 1 resident), then 16 clock64 phase stamps per iteration
 * (block 0, thread 0).  cap >= 1032; *n = 0 when nothing was traced. */
silk_status silk_debug_cg_trace(const silk_world* w, uint32_t handle, int64_t* trace,
                               int64_t cap, int32_t* n);

/* --- Inspection entry points used by the parity tests ------------------- */
/* Solver-order permutation (original -> solver) and partition offsets. */
silk_status silk_debug_cloth_partition(const silk_world* w, uint32_t handle,
                                       int32_t* perm, int64_t perm_len,
                                       int32_t* part_offsets,
                                       int64_t offsets_cap, int32_t* nparts);
/* Scalar system matrix L (H = L (x) I3) as dense row-major, solver order. */
silk_status silk_debug_cloth_matrix(const silk_world* w, uint32_t handle,
                                    double* dense, int64_t n_len);
/* Fine MAS level of the last factorisation (MASPreconditioner::factorize,
 * mas_preconditioner.cu:903-965): the FP32 bank inverses (packed upper
 * triangle, 528 floats per bank, banks in partition order, slot = solver
 * index - first vertex of the bank) and the diagonal the ADMM adds to L
 * (nv floats, solver order), the bank matrix being L + diag restricted to
 * the bank. */
silk_status silk_debug_mas_fine(const silk_world* w, uint32_t handle, float* inverses,
                                int64_t inverses_len, float* diag, int64_t diag_len);
/* Refit every collider to (t0 = current state, t1 = current + disp) where
 * disp is per cloth in original vertex order, concatenated. */
silk_status silk_debug_refit(silk_world* w, const float* disp,
                             int64_t disp_len);
/* Broadphase candidates of the current refit: rows of
 * (kind, object_a, index_a, object_b, index_b); returns count in *n. */
silk_status silk_debug_candidates(silk_world* w, int32_t* out, int64_t cap,
                                  int32_t* n);
/* DCD contact keys at collider time t: rows of (type, obj_a, obj_b, i0..i3)
 * sorted; count in *n. */
silk_status silk_debug_dcd(silk_world* w, float t, float activation,
                           int32_t* keys, int64_t cap, int32_t* n);
/* Active contact set of the last solver_step (the contacts DCD activated at
 * the start of the step and after each rollback, deduplicated by the
 * reference's canonical key, contact_constraints.cu:440-453): rows of
 * (type, obj_a, obj_b, i0..i3) in canonical order; *n = total count (rows
 * beyond cap are not written). */
silk_status silk_debug_contacts(silk_world* w, int32_t* keys, int64_t cap, int32_t* n);
/* Minimum time of impact over the current refit.  prune = 1 lets searches
 * stop once they cannot lower the minimum (the solver step's mode: same
 * minimum, n_hits then counts completed searches only). */
silk_status silk_debug_min_toi(silk_world* w, float time_start,
                               float max_time, float min_separation,
                               int32_t prune, float* toi, int32_t* n_queries,
                               int32_t* n_hits);

/* --- Host-side setup (no GPU needed) ------------------------------------ */
/* Vertex partition used as the MAS banks: connected parts of <= 32
 * vertices (replaces MeshPartition, backend/cuda/mesh_partition.cu:56-105,
 * whose KaMinPar/METIS partitioner is not available here). */
silk_status silk_partition_mesh(const float* verts, int64_t verts_len,
                                const int32_t* faces, int64_t faces_len,
                                int32_t* perm, int32_t* part_offsets,
                                int64_t offsets_cap, int32_t* nparts);
/* Entry order of one MAS bank's 32 matrix rows in the resident CG kernel's
 * ELL slice (no reference counterpart; inspection entry point for the
 * tests): row l holds cols/vals[row_ptr[l] .. row_ptr[l + 1]) (a column < 0
 * is shared-memory slot -1 - column), width >= the longest row, slot0 the
 * bank's first slot; out_cols/out_vals receive width x 32 entries, round j
 * of row l at [j * 32 + l] (padding: value 0). */
silk_status silk_schedule_bank_rows(const int32_t* row_ptr, const int32_t* cols,
                                    const int32_t* vals, int32_t width, int32_t slot0,
                                    int32_t* out_cols, int32_t* out_vals);
/* Static assembly of one cloth in solver order (ClothAssemblyL2Cache +
 * ClothAssemblyL1Cache, cloth_assembly_l2_cache.cpp:71-136,
 * cloth_assembly_l1_cache.cu:16-97): dense scalar matrix L (nv x nv, may be
 * NULL), mass (nv), contact weight (nv), bending rhs (3 nv). */
silk_status silk_assemble_cloth_host(const silk_cloth_config* cloth,
                                     const float* verts, int64_t verts_len,
                                     const int32_t* faces, int64_t faces_len,
                                     float dt, double* dense_L, double* mass,
                                     double* contact_weight,
                                     double* bending_rhs);

/* --- Standalone operators ---------------------------------------------- */
/* Tight-Inclusion CCD of n queries on the GPU.  x: n x 24 floats (4 points
 * at t0 then 4 at t1; point-triangle: point first).  Writes hit (0/1) and
 * the time of impact (lower bound of the accepted interval; the refined
 * minimum-separation interval when the first starts at 0). */
silk_status silk_ccd_batch(int32_t is_vertex_face, const float* x, int64_t n,
                           const float* err3, const float* min_separation,
                           float tolerance, int32_t max_iter, float max_time,
                           int32_t* hit, float* toi, float* t_upper);
/* The contact Gauss-Seidel's Coulomb projection run on the GPU for n
 * (free displacement u, unit normal, friction coefficient) triples: the
 * device function every contact projection of a step uses
 * (solve_coulomb_contact, contact_constraints.cu:391-411); out receives n x 3
 * projected displacements.  Inspection entry point for the known-answer
 * tests of test/friction_contact_test.cu:23-92. */
silk_status silk_debug_coulomb(const float* u, const float* normal, const float* friction,
                               int64_t n, float* out);
/* Contact colouring of n contacts given 4 vertex ids each (-1 = immovable)
 * and 64-bit priorities: greedy colouring in decreasing priority order. */
silk_status silk_color_contacts(const int32_t* verts4, const uint64_t* prio,
                                int64_t n, int32_t* colors, int32_t* ncolors);

/* --- Learned CG warm start (no counterpart in the reference) ------------ */
/* Per-vertex MLP 13 -> 64 -> 64 -> 64 -> 3 (GELU, BF16 weights and layer
 * inputs on the tensor cores, FP32 accumulation) that predicts the solution
 * of the first CG solve of every outer iteration from the vertex's inertial
 * offset, last two step displacements, 1-ring mean displacement and pin
 * flag.  The prediction is only offered: the CG kernel starts from it when its
 * residual is smaller than the plain start's, and always stops at
 * rel_tol^2 x the plain start's residual norm.  Parameters are one FP32
 * vector of SILK_MLP_PARAMS floats: W1 (16x64), b1, W2 (64x64), b2, W3, b3,
 * W4 (64x8), b4 (8), feature mean (16), feature std (16), output scale (8);
 * weights row-major (input, output). */
#define SILK_MLP_PARAMS 9968
/* Load trained models into the world (NULL disables them); used when the
 * solver option learned_warm_start is 1.  n = SILK_MLP_PARAMS: the
 * first-solve model; n = 2 * SILK_MLP_PARAMS: the first-solve model followed
 * by the iterate model, the same network over 13 features of the last three
 * ADMM iterates x_k, x_(k-1), x_(k-2) (x_k - x_(k-1), x_(k-1) - x_(k-2), the
 * 1-ring means of both, the pin flag, all over sigma = the RMS of
 * x_k - x_(k-1) over the vertices) that predicts (x_(k+1) - x_k) / sigma;
 * x_k + sigma * prediction is offered to the solve for x_(k+1) like the
 * first-solve start (taken only where it lowers the residual, the plain
 * start's residual stays the stopping reference). */
silk_status silk_set_warm_start_model(silk_world* w, const float* params, int64_t n);
/* Iterate-model training samples of the last step (solver option
 * capture_samples bit 2): up to cap rows of 16 features (13 used) and 4
 * targets (3 used, (x_(k+1) - x_k) / sigma); *n = rows written. */
silk_status silk_get_iterate_samples(silk_world* w, float* features, float* targets, int64_t cap,
                                     int32_t* n);
/* Training samples of the last step (solver option capture_samples = 1):
 * per vertex 16 features (13 used) and 4 targets (3 used: first CG solution
 * minus the inertial prediction, over the step scale dt^2 |g|), in the
 * solver's vertex order; *valid = 0 when the last step recorded none. */
silk_status silk_get_warm_start_samples(const silk_world* w, uint32_t handle,
                                        float* features, float* targets,
                                        int64_t nverts, int32_t* valid);
/* Model outputs (n x 3, normalised units) of n feature rows (n x 16). */
silk_status silk_mlp_forward(const float* params, const float* features, int64_t n,
                             float* out);
/* Mean squared error against targets (n x 4, 3 used, already divided by
 * the step scale and the output scale) and its gradient (SILK_MLP_PARAMS
 * floats, statistics entries zero). */
silk_status silk_mlp_loss_grad(const float* params, const float* features,
                               const float* targets, int64_t n, float* grad,
                               double* loss);
/* Adam training on the GPU: `steps` updates on batches of `batch` samples
 * drawn with replacement (batch <= 0 or >= n: full batch); params updated in
 * place; loss_history (steps floats, may be NULL) gets each step's loss. */
silk_status silk_mlp_train(float* params, const float* features, const float* targets,
                           int64_t n, int32_t steps, int32_t batch, float lr,
                           uint64_t seed, float* loss_history);

/* --- CCD batch that allocates nothing ----------------------------------- */
/* No counterpart in the reference (its narrowphase, narrowphase.cu and
 * ccd.cpp, runs on host cores).  Same queries and results as
 * silk_ccd_batch, for callers that must not allocate device memory: hosts
 * whose device memory is owned by a pool or arena with a fixed budget (an
 * allocation outside it can fail or evict), and real-time loops in which
 * cudaMalloc / cudaFree would synchronise the device and stall other
 * streams.  The call performs no cudaMalloc, cudaFree or other allocating
 * routine; its working memory is one static device array of 10,489,088
 * bytes created with the library on each device that loads it.
 *
 * Buffers x (n x 24 floats), min_separation (n), hit (n), toi (n) and
 * t_upper (n, may be NULL) are device (or managed) memory of the CURRENT
 * device, 4-byte aligned; err3 (3 floats) and n_spilled (may be NULL; the
 * number of queries that needed the large second-pass storage) are host
 * memory.  Work is issued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and the call returns after it has finished.
 *
 * Limits: n <= SILK_CCD_NOALLOC_MAX_QUERIES and
 * 1 <= max_iter <= SILK_CCD_NOALLOC_MAX_ITER; outside them the call returns
 * SILK_ERR_INVALID_CONFIG before touching the device.  Host (non-device)
 * or misaligned buffers, NULL pointers and n < 0 also give
 * SILK_ERR_INVALID_CONFIG, and so does a `stream` that is being captured
 * (the call reads its counters back and synchronises the stream, so it
 * refuses such a stream before queuing anything on it); a CUDA error gives
 * SILK_ERR_UNKNOWN.  If a query's search ever needed more pending boxes than
 * its second-pass storage region holds (not reachable within the limits:
 * a search keeps at most max_iter + 2 pending boxes), that query is reported
 * as a hit at time 0 with t_upper = max_time and the call returns
 * SILK_ERR_UNKNOWN after writing every other query's result.
 *
 * The first call on each device (any n, 0 included) looks up the scratch
 * array's address, which loads the library's kernels onto that device; make
 * that first call before any stream capture begins.  Each call zeroes the
 * scratch counters itself, so nothing has to be cleared between calls.  All
 * calls on one device share the one scratch array: overlapping calls would
 * race on it, so calls on the same device from several host threads are
 * serialised by a lock inside the library and each holds it until its work
 * on the device has finished, also when it returns an error after queuing
 * work.  The scratch address is looked up once per device and kept for the
 * life of the process: do not call this entry point again on a device after
 * cudaDeviceReset has destroyed the context it was looked up in. */
#define SILK_CCD_NOALLOC_MAX_QUERIES (1 << 20)
#define SILK_CCD_NOALLOC_MAX_ITER 4096
silk_status silk_ccd_batch_noalloc(int32_t is_vertex_face, const float* x,
                                   int64_t n, const float* err3,
                                   const float* min_separation, float tolerance,
                                   int32_t max_iter, float max_time,
                                   int32_t* hit, float* toi, float* t_upper,
                                   void* stream, int32_t* n_spilled);

#ifdef __cplusplus
}
#endif

#endif /* SILK_B200_H */
