// Device views and kernel launchers of the ADMM cloth solver.
#pragma once

#include "common.cuh"

namespace silkb {

// Per-vertex / per-face arrays of every cloth of a world, concatenated in
// solver order.  Vectors of 3 DoF are float4 with w = 0 (16-byte aligned
// loads and stores).
struct SolverView {
  int nv = 0;  // total cloth vertices
  int nf = 0;  // total cloth faces
  float dt = 0.0f;
  float4 acc{};  // constant acceleration
  // State.
  float4* x = nullptr;       // current ADMM iterate (inner state)
  const float4* prev = nullptr;    // state at step start
  const float4* prev_v = nullptr;  // damped velocity at step start
  // Static per vertex.
  const float* mass = nullptr;          // density * Voronoi area
  const float4* bending_rhs = nullptr;  // k_b C^T W C x_rest
  // Faces.
  const int4* faces = nullptr;    // global vertex ids (w unused)
  const float4* B0 = nullptr;     // chart row 0 (xyz) + sqrt(area) (w)
  const float4* B1 = nullptr;     // chart row 1 (xyz) + penalty rho (w)
  float4* zu = nullptr;           // 3 per face: z0..z5, u0..u5
  float4* zold = nullptr;         // 2 per face: previous z
  const int* vf_off = nullptr;    // vertex -> incident (face << 2 | corner)
  const int* vf_list = nullptr;
  // Pins (equality constraints, equality_constraints.cu).
  const unsigned char* pin_flag = nullptr;
  const float4* pin_target = nullptr;
  float4* pin_lambda = nullptr;
  // Contacts (per vertex weight; p = auxiliary position, eta multiplier).
  const float* contact_w = nullptr;
  float4* contact_p = nullptr;
  float4* contact_p_prev = nullptr;
  float4* contact_eta = nullptr;
  // Assembled right-hand side / dynamic diagonal of the next x-update.
  float* lhs = nullptr;
  float4* rhs = nullptr;
  float4* inertia = nullptr;  // -x_prev/dt^2 - v_prev/dt - a
  // AdmmControl::done of the running ADMM solve: the per-iteration kernels
  // (face step, contact init, vertex step) return at entry when it is set.
  const int* skip = nullptr;
};

// ADMM reduction slots (double partial sums per block).
enum AdmmSlot {
  kPrimalNorm2 = 0,
  kPrimalScaleX2 = 1,
  kPrimalScaleAux2 = 2,
  kDualNorm2 = 3,
  kDualCur2 = 4,
  kDualPrev2 = 5,
  kNonFinite = 6,
  kAdmmSlots = 8
};

struct AdmmControl {
  // Written by the convergence test, read by the host every few iterations.
  int converged;
  int diverged;
  float next_rel_tol;
  float primal_norm;
  float dual_norm;
  float init_primal;
  float init_dual;
  float ratio;
  int iteration;
  // Set with converged or diverged: the iterations the host enqueued beyond
  // this one find it at entry and do nothing.
  int done;
  // Blocks of the running vertex step that have stored their partials; the
  // last one runs the convergence test and sets it back to 0.
  unsigned ticket;
  int pad[5];
};
static_assert(sizeof(AdmmControl) == 64, "one control block of 64 bytes");

void launch_compute_inertia(const SolverView& s, cudaStream_t st);
// Face step (local elastic projection, residual partials) of one ADMM
// iteration; with contact_init, the same launch also sets the contacts'
// auxiliary positions (initialize_aux).
void launch_face_step(const SolverView& s, double* partials, int nblocks, bool contact_init,
                      cudaStream_t st);
int face_step_blocks(int nf);
int vertex_step_blocks(int nv);
struct AdmmFinalizeArgs {
  const double* face_partials;
  int face_blocks;
  double* vertex_partials;
  int vertex_blocks;
  int dof_primal_static;     // 6 * faces + pinned dof
  const int* contact_active_dof;  // device scalar (may be null)
  int state_dof;
  float abs_tol, rel_tol;
  float init_lin_rel, lin_rel_min, lin_rel_max, fixed_rel;
  int iteration;  // 0: the first iteration, which has no convergence test
  AdmmControl* ctl;
  const int* cg_fail = nullptr;  // set when a CG barrier wait gave up
};
// Vertex step (multiplier updates, dual residual, next system's right-hand
// side) of one ADMM iteration on fa.vertex_blocks blocks; its last block to
// finish runs the iteration's convergence test into fa.ctl.
void launch_vertex_step(const SolverView& s, const AdmmFinalizeArgs& fa, cudaStream_t st);
void launch_enforce(const SolverView& s, cudaStream_t st);
void launch_predict(int nv, float dt, float4 acc, const float4* x,
                    const float4* v, float4* out, cudaStream_t st);
// ext = 2 x - prev where valid, then prev = x (ADMM-extrapolated CG start).
void launch_extrapolate(int nv, bool valid, const float4* x, float4* prev, float4* ext,
                        cudaStream_t st);
void launch_velocity(int nv, float dt, const float4* a, const float4* b,
                     float4* v, cudaStream_t st);
void launch_mix(int nv, float w, const float4* a, float4* b, cudaStream_t st);
void launch_damp(int nv, const float* damp, const float4* v, float4* out,
                 cudaStream_t st);

}  // namespace silkb
