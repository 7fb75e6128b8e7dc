// ADMM projective-dynamics kernels: per-face local projection, per-vertex
// multiplier updates / residuals / right-hand-side assembly, convergence.
//
// Reference: backend/cuda/solver/admm_solver.cu:86-342,
// cloth_admm_helper.cu:19-271, equality_constraints.cu:14-125,
// contact_constraints.cu:203-217 and :302-374, main_loop.cu:78-120.
//
// Layout: the system matrix of a cloth is L (x) I3 (every 3x3 block of
// k_e J^T W J + k_b C^T W C (x) I3 is a multiple of I3 because J = B (x) I3),
// so each face keeps only its 2x3 chart operator B instead of the 6x9 J.
#include "solver_kernels.cuh"

namespace silkb {

thread_local long long g_launch_count = 0;

namespace {

constexpr float kPinPenalty = 1e4f;   // pin_constraints.cu:101
constexpr float kMaxMultiplier = 1e8f;  // ADMMSolver::max_lagrange_mul

template <int N>
__device__ void block_reduce_store(double (&v)[N], double* out) {
  __shared__ double sh[N][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double a = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) sh[k][warp] = a;
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double a = lane < nw ? sh[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) out[k] = a;
    }
  }
}

// Clamped projection of a 3x2 deformation gradient onto singular values in
// [lo, hi] (cloth_admm_helper.cu:19-51).  The right singular vectors come
// from a Jacobi rotation that diagonalises F^T F; the left ones from F V.
__device__ void clamp_projection(const float (&y)[6], float lo, float hi,
                                 float (&out)[6]) {
  float g11 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
  float g22 = y[3] * y[3] + y[4] * y[4] + y[5] * y[5];
  float g12 = y[0] * y[3] + y[1] * y[4] + y[2] * y[5];
  float theta = 0.5f * atan2f(2.0f * g12, g11 - g22);
  float s, c;
  sincosf(theta, &s, &c);
  float v1x = c, v1y = s, v2x = -s, v2y = c;
  float u1[3], u2[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    u1[i] = y[i] * v1x + y[3 + i] * v1y;
    u2[i] = y[i] * v2x + y[3 + i] * v2y;
  }
  float s1 = sqrtf(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  float s2 = sqrtf(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
  if (s1 < s2) {
    float t = s1;
    s1 = s2;
    s2 = t;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float q = u1[i];
      u1[i] = u2[i];
      u2[i] = q;
    }
    float a = v1x, b = v1y;
    v1x = v2x;
    v1y = v2y;
    v2x = a;
    v2y = b;
  }
  if (s1 > 0.0f) {
    float inv = 1.0f / s1;
#pragma unroll
    for (int i = 0; i < 3; ++i) u1[i] *= inv;
  } else {
    u1[0] = 1.0f;
    u1[1] = 0.0f;
    u1[2] = 0.0f;
  }
  if (s2 > 1e-7f * s1) {
    float inv = 1.0f / s2;
#pragma unroll
    for (int i = 0; i < 3; ++i) u2[i] *= inv;
  } else {
    // Collapsed triangle: complete u2 with a unit vector orthogonal to u1.
    float a0 = fabsf(u1[0]) < 0.9f ? 1.0f : 0.0f;
    float a1 = fabsf(u1[0]) < 0.9f ? 0.0f : 1.0f;
    float d = a0 * u1[0] + a1 * u1[1];
    float w0 = a0 - d * u1[0], w1 = a1 - d * u1[1], w2 = -d * u1[2];
    float inv = rsqrtf(w0 * w0 + w1 * w1 + w2 * w2);
    u2[0] = w0 * inv;
    u2[1] = w1 * inv;
    u2[2] = w2 * inv;
  }
  float c1 = fminf(fmaxf(s1, lo), hi), c2 = fminf(fmaxf(s2, lo), hi);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    out[i] = c1 * u1[i] * v1x + c2 * u2[i] * v2x;
    out[3 + i] = c1 * u1[i] * v1y + c2 * u2[i] * v2y;
  }
}

__global__ void inertia_kernel(SolverView s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.nv) return;
  float4 x = s.prev[i], v = s.prev_v[i];
  float dt2 = s.dt * s.dt;
  float4 o;
  o.x = -x.x / dt2 - v.x / s.dt - s.acc.x;
  o.y = -x.y / dt2 - v.y / s.dt - s.acc.y;
  o.z = -x.z / dt2 - v.z / s.dt - s.acc.z;
  o.w = 0.0f;
  s.inertia[i] = o;
}

// initialize_aux (contact_constraints.cu:203-215): p <- x - eta / w.
__device__ __forceinline__ void contact_init(const SolverView& s, int i) {
  if (i >= s.nv) return;
  float w = s.contact_w[i];
  float4 p = s.contact_p[i];
  s.contact_p_prev[i] = p;
  float4 x = s.x[i];
  if (w > 0.0f) {
    float4 e = s.contact_eta[i];
    p = make_float4(x.x - e.x / w, x.y - e.y / w, x.z - e.z / w, 0.f);
  } else {
    p = x;
  }
  s.contact_p[i] = p;
}

// solve_and_update_elastic_aux (cloth_admm_helper.cu:81-201) without the
// per-vertex dual scatter, which the vertex kernel gathers instead.  Blocks
// from face_blocks on initialise the contacts' auxiliary positions instead
// (they touch none of the faces' arrays), so one launch does both.
__global__ void __launch_bounds__(THREADS) face_step_kernel(SolverView s, double* partials,
                                                            int face_blocks) {
  if (s.skip && *s.skip) return;  // the ADMM solve already ended
  if ((int)blockIdx.x >= face_blocks) {
    contact_init(s, ((int)blockIdx.x - face_blocks) * blockDim.x + threadIdx.x);
    return;
  }
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[3] = {0.0, 0.0, 0.0};
  if (f < s.nf) {
    int4 F = s.faces[f];
    float4 b0 = s.B0[f], b1 = s.B1[f];
    float w = b0.w, rho = b1.w;
    float4 xa = s.x[F.x], xb = s.x[F.y], xc = s.x[F.z];
    float Sx[6];
    Sx[0] = b0.x * xa.x + b0.y * xb.x + b0.z * xc.x;
    Sx[1] = b0.x * xa.y + b0.y * xb.y + b0.z * xc.y;
    Sx[2] = b0.x * xa.z + b0.y * xb.z + b0.z * xc.z;
    Sx[3] = b1.x * xa.x + b1.y * xb.x + b1.z * xc.x;
    Sx[4] = b1.x * xa.y + b1.y * xb.y + b1.z * xc.y;
    Sx[5] = b1.x * xa.z + b1.y * xb.z + b1.z * xc.z;
    float4 q0 = s.zu[3 * f], q1 = s.zu[3 * f + 1], q2 = s.zu[3 * f + 2];
    float z[6] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
    float u[6] = {q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
    float inv = 1.0f / (rho * w);
    float y[6], proj[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) y[r] = Sx[r] + inv * u[r];
    clamp_projection(y, 0.9f, 1.1f, proj);
    // Stiffness k equals the penalty rho (cloth_assembly_l1_cache.cu:24).
    float ratio = rho / (rho + rho);
    float zn[6], un[6];
    float pn = 0.f, px = 0.f, pa = 0.f;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      zn[r] = (1.0f - ratio) * y[r] + ratio * proj[r];
      float pr = w * (Sx[r] - zn[r]);
      pn += pr * pr;
      px += (w * Sx[r]) * (w * Sx[r]);
      pa += (w * zn[r]) * (w * zn[r]);
      float d = w * rho * Sx[r] + (-w * rho) * zn[r];
      un[r] = fminf(fmaxf(u[r] + d, -kMaxMultiplier), kMaxMultiplier);
    }
    acc[0] = pn;
    acc[1] = px;
    acc[2] = pa;
    s.zold[2 * f] = make_float4(z[0], z[1], z[2], z[3]);
    s.zold[2 * f + 1] = make_float4(z[4], z[5], 0.f, 0.f);
    s.zu[3 * f] = make_float4(zn[0], zn[1], zn[2], zn[3]);
    s.zu[3 * f + 1] = make_float4(zn[4], zn[5], un[0], un[1]);
    s.zu[3 * f + 2] = make_float4(un[2], un[3], un[4], un[5]);
  }
  block_reduce_store<3>(acc, partials + (size_t)blockIdx.x * kAdmmSlots);
}

__device__ void admm_finalize(const AdmmFinalizeArgs& a);

// Per-vertex part of one ADMM iteration: pin multiplier update and primal
// residual (equality_constraints.cu:49-104), contact multiplier update
// (contact_constraints.cu:320-374), dual residual gathered over incident
// faces, finiteness check, and assembly of the next x-update system
// (cloth_admm_helper.cu:203-271, equality_constraints.cu:66-80,
// contact_constraints.cu:302-318).  The last block to store its partials
// (a ticket in the control block) then runs the iteration's convergence
// test, from iteration 1 on (fa.iteration > 0).
__global__ void __launch_bounds__(THREADS) vertex_step_kernel(SolverView s,
                                                              AdmmFinalizeArgs fa) {
  if (s.skip && *s.skip) return;  // the ADMM solve already ended
  double* partials = fa.vertex_partials;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < s.nv) {
    float4 x = s.x[i];
    float xv[3] = {x.x, x.y, x.z};
    float lhs = s.mass[i] / (s.dt * s.dt);
    float4 br = s.bending_rhs[i], in = s.inertia[i];
    float m = s.mass[i];
    float rhs[3] = {br.x - m * in.x, br.y - m * in.y, br.z - m * in.z};
    float pn = 0.f, px = 0.f, pa = 0.f;
    if (s.pin_flag[i]) {
      float4 t = s.pin_target[i], l = s.pin_lambda[i];
      float tv[3] = {t.x, t.y, t.z}, lv[3] = {l.x, l.y, l.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lv[a] = fminf(fmaxf(lv[a] + kPinPenalty * (xv[a] - tv[a]), -kMaxMultiplier),
                      kMaxMultiplier);
        float d = xv[a] - tv[a];
        pn += d * d;
        px += xv[a] * xv[a];
        pa += tv[a] * tv[a];
        rhs[a] += kPinPenalty * tv[a] - lv[a];
      }
      lhs += kPinPenalty;
      s.pin_lambda[i] = make_float4(lv[0], lv[1], lv[2], 0.f);
    }
    float dual[3] = {0, 0, 0}, dcur[3] = {0, 0, 0}, dprev[3] = {0, 0, 0};
    float w = s.contact_w[i];
    if (w > 0.0f) {
      float4 p = s.contact_p[i], pp = s.contact_p_prev[i], e = s.contact_eta[i];
      float pv[3] = {p.x, p.y, p.z}, ppv[3] = {pp.x, pp.y, pp.z},
            ev[3] = {e.x, e.y, e.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float pr = xv[a] - pv[a];
        ev[a] += w * (pv[a] - xv[a]);
        pn += pr * pr;
        dual[a] += w * (pv[a] - ppv[a]);
        dcur[a] += ev[a];
        dprev[a] += ev[a];
        rhs[a] += w * pv[a] + ev[a];
      }
      lhs += w;
      s.contact_eta[i] = make_float4(ev[0], ev[1], ev[2], 0.f);
    }
    float erhs[3] = {0, 0, 0}, ecur[3] = {0, 0, 0}, eprev[3] = {0, 0, 0};
    for (int k = s.vf_off[i]; k < s.vf_off[i + 1]; ++k) {
      int code = s.vf_list[k];
      int f = code >> 2, corner = code & 3;
      float4 b0 = s.B0[f], b1 = s.B1[f];
      float bk0 = corner == 0 ? b0.x : (corner == 1 ? b0.y : b0.z);
      float bk1 = corner == 0 ? b1.x : (corner == 1 ? b1.y : b1.z);
      float fw = b0.w, rho = b1.w;
      float4 q0 = s.zu[3 * f], q1 = s.zu[3 * f + 1], q2 = s.zu[3 * f + 2];
      float4 o0 = s.zold[2 * f], o1 = s.zold[2 * f + 1];
      float z[6] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
      float u[6] = {q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
      float zo[6] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y};
      float sc = rho * fw * fw;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float stz = bk0 * z[a] + bk1 * z[3 + a];
        float stu = bk0 * u[a] + bk1 * u[3 + a];
        float stzo = bk0 * zo[a] + bk1 * zo[3 + a];
        erhs[a] += -fw * stu + sc * stz;
        ecur[a] += sc * stz;
        eprev[a] += sc * stzo;
      }
    }
    float d2 = 0.f, c2 = 0.f, q2s = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float dd = dual[a] + (ecur[a] - eprev[a]);
      float cc = dcur[a] + ecur[a];
      float qq = dprev[a] + eprev[a];
      d2 += dd * dd;
      c2 += cc * cc;
      q2s += qq * qq;
      rhs[a] += erhs[a];
    }
    acc[0] = pn;
    acc[1] = px;
    acc[2] = pa;
    acc[3] = d2;
    acc[4] = c2;
    acc[5] = q2s;
    acc[6] = (isfinite(x.x) && isfinite(x.y) && isfinite(x.z)) ? 0.0 : 1.0;
    s.lhs[i] = lhs;
    s.rhs[i] = make_float4(rhs[0], rhs[1], rhs[2], 0.f);
  }
  block_reduce_store<7>(acc, partials + (size_t)blockIdx.x * kAdmmSlots);
  // Thread 0 stored this block's partials: fence them, then take a ticket.
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&fa.ctl->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) fa.ctl->ticket = 0u;  // for the next iteration's launch
  if (fa.iteration > 0) admm_finalize(fa);
}

// Convergence test of one ADMM iteration (admm_solver.cu:209-330): the block
// sums the face and vertex partials slot by slot in a fixed order (lanes
// stride the blocks, then a shuffle tree) and thread 0 updates the control
// block.  Partials are read from L2: the vertex partials come from other
// blocks of the launch that runs this.
__device__ void admm_finalize(const AdmmFinalizeArgs& a) {
  __shared__ double sh[kAdmmSlots][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // warp k < 3 sums face slot k, warps 3.. sum vertex slots.
  for (int slot = warp; slot < 7; slot += blockDim.x >> 5) {
    double s = 0.0;
    if (slot < 3)
      for (int b = lane; b < a.face_blocks; b += 32)
        s += __ldcg(a.face_partials + (size_t)b * kAdmmSlots + slot);
    for (int b = lane; b < a.vertex_blocks; b += 32)
      s += __ldcg(a.vertex_partials + (size_t)b * kAdmmSlots + slot);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[slot][0] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  AdmmControl* c = a.ctl;
  double pn2 = sh[kPrimalNorm2][0], px2 = sh[kPrimalScaleX2][0],
         pa2 = sh[kPrimalScaleAux2][0];
  double d2 = sh[kDualNorm2][0], c2 = sh[kDualCur2][0], q2 = sh[kDualPrev2][0];
  c->iteration = a.iteration;
  if (sh[kNonFinite][0] > 0.0 || (a.cg_fail && *a.cg_fail)) {
    c->diverged = 1;
    c->converged = 0;
    c->done = 1;
    return;
  }
  float pnorm = sqrtf((float)pn2);
  if (a.iteration == 1) c->init_primal = pnorm;
  int dof = a.dof_primal_static + (a.contact_active_dof ? *a.contact_active_dof : 0);
  float peps = (float)sqrt((double)dof) * a.abs_tol +
               fmaxf(sqrtf((float)px2), sqrtf((float)pa2)) * a.rel_tol;
  float dnorm = sqrtf((float)d2);
  if (a.iteration == 1) c->init_dual = dnorm;
  float deps = (float)sqrt((double)a.state_dof) * a.abs_tol +
               fmaxf(sqrtf((float)c2), sqrtf((float)q2)) * a.rel_tol;
  float ratio = fmaxf(pnorm / fmaxf(c->init_primal, a.abs_tol),
                      dnorm / fmaxf(c->init_dual, a.abs_tol));
  c->ratio = ratio;
  c->primal_norm = pnorm;
  c->dual_norm = dnorm;
  c->converged = (pnorm <= peps && dnorm <= deps) ? 1 : 0;
  c->diverged = 0;
  c->done = c->converged;
  float rel = fminf(fmaxf(a.init_lin_rel * ratio, a.lin_rel_min), a.lin_rel_max);
  c->next_rel_tol = a.fixed_rel > 0.0f ? a.fixed_rel : rel;
}

// pins.enforce + contacts.project (admm_solver.cu:333-339).
__global__ void enforce_kernel(SolverView s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.nv) return;
  if (s.pin_flag[i]) s.x[i] = s.pin_target[i];
  if (s.contact_w[i] > 0.0f) s.x[i] = s.contact_p[i];
}

__global__ void predict_kernel(int nv, float dt, float4 acc, const float4* x,
                               const float4* v, float4* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float4 a = x[i], b = v[i];
  float nx = 1.0f * a.x + dt * b.x, ny = 1.0f * a.y + dt * b.y,
        nz = 1.0f * a.z + dt * b.z;
  float dt2 = dt * dt;
  out[i] = make_float4(1.0f * nx + dt2 * acc.x, 1.0f * ny + dt2 * acc.y,
                       1.0f * nz + dt2 * acc.z, 0.f);
}

__global__ void velocity_kernel(int nv, float dt, const float4* a,
                                const float4* b, float4* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float4 p = a[i], q = b[i];
  v[i] = make_float4((p.x - q.x) / dt, (p.y - q.y) / dt, (p.z - q.z) / dt, 0.f);
}

// Extrapolated CG start from the last two ADMM iterates of one ADMM solve:
// ext = 2 x_k - x_(k-1) when prev holds x_(k-1) (valid), then prev = x_k.
__global__ void extrapolate_kernel(int nv, int valid, const float4* x, float4* prev,
                                   float4* ext) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float4 p = x[i];
  if (valid) {
    float4 q = prev[i];
    ext[i] = make_float4(p.x + (p.x - q.x), p.y + (p.y - q.y), p.z + (p.z - q.z), 0.f);
  }
  prev[i] = p;
}

// out = w * a + (1 - w) * b with the second term in double (main_loop.cu:111).
__global__ void mix_kernel(int nv, float w, const float4* a, float4* b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float4 p = a[i], q = b[i];
  double r = 1.0 - (double)w;
  b[i] = make_float4((float)((double)(w * p.x) + r * q.x),
                     (float)((double)(w * p.y) + r * q.y),
                     (float)((double)(w * p.z) + r * q.z), 0.f);
}

__global__ void damp_kernel(int nv, const float* damp, const float4* v,
                            float4* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float d = damp[i];
  float4 a = v[i];
  out[i] = make_float4(d * a.x, d * a.y, d * a.z, 0.f);
}

}  // namespace

int face_step_blocks(int nf) { return div_up(nf > 0 ? nf : 1, THREADS); }
int vertex_step_blocks(int nv) { return div_up(nv > 0 ? nv : 1, THREADS); }

void launch_compute_inertia(const SolverView& s, cudaStream_t st) {
  if (s.nv == 0) return;
  inertia_kernel<<<div_up(s.nv, THREADS), THREADS, 0, st>>>(s);
  SILK_LAUNCHED();
}

void launch_face_step(const SolverView& s, double* partials, int nblocks, bool contact_init,
                      cudaStream_t st) {
  const int init_blocks = contact_init ? div_up(s.nv, THREADS) : 0;
  face_step_kernel<<<nblocks + init_blocks, THREADS, 0, st>>>(s, partials, nblocks);
  SILK_LAUNCHED();
}

void launch_vertex_step(const SolverView& s, const AdmmFinalizeArgs& fa, cudaStream_t st) {
  vertex_step_kernel<<<fa.vertex_blocks, THREADS, 0, st>>>(s, fa);
  SILK_LAUNCHED();
}

void launch_enforce(const SolverView& s, cudaStream_t st) {
  enforce_kernel<<<div_up(s.nv, THREADS), THREADS, 0, st>>>(s);
  SILK_LAUNCHED();
}

void launch_predict(int nv, float dt, float4 acc, const float4* x,
                    const float4* v, float4* out, cudaStream_t st) {
  predict_kernel<<<div_up(nv, THREADS), THREADS, 0, st>>>(nv, dt, acc, x, v, out);
  SILK_LAUNCHED();
}

void launch_velocity(int nv, float dt, const float4* a, const float4* b,
                     float4* v, cudaStream_t st) {
  velocity_kernel<<<div_up(nv, THREADS), THREADS, 0, st>>>(nv, dt, a, b, v);
  SILK_LAUNCHED();
}

void launch_extrapolate(int nv, bool valid, const float4* x, float4* prev, float4* ext,
                        cudaStream_t st) {
  extrapolate_kernel<<<div_up(nv, THREADS), THREADS, 0, st>>>(nv, valid ? 1 : 0, x, prev, ext);
  SILK_LAUNCHED();
}

void launch_mix(int nv, float w, const float4* a, float4* b, cudaStream_t st) {
  mix_kernel<<<div_up(nv, THREADS), THREADS, 0, st>>>(nv, w, a, b);
  SILK_LAUNCHED();
}

void launch_damp(int nv, const float* damp, const float4* v, float4* out,
                 cudaStream_t st) {
  damp_kernel<<<div_up(nv, THREADS), THREADS, 0, st>>>(nv, damp, v, out);
  SILK_LAUNCHED();
}

}  // namespace silkb
