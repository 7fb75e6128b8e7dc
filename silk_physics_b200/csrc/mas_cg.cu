// MAS factorisation and the persistent PCG solve.
//
// Reference: backend/cuda/solver/mas_preconditioner.cu:489-989 (coarse
// matrices, packed inverses, multilevel apply) and mas_cg_solver.cu:30-311
// (PCG with the same stopping rules: rr <= abs^2, rr <= rel^2 rr0, max_iter,
// alpha/beta guarded by |denominator| < 1e-20, at least one iteration).
//
// The B200 design differs from the reference in three ways:
//  * bank matrices are 32x32 scalar blocks (the system is L (x) I3), built
//    and inverted in FP64 from static gather plans (no atomics), and stored
//    packed in FP32 or BF16;
//  * the whole CG loop, including every MAS level, runs inside one
//    cooperative kernel whose phases are separated by a grid barrier with a
//    bounded spin (no host round trip, no graph rebuild per solve);
//  * reductions are FP64 and deterministic (per-block partials summed in a
//    fixed order by every block);
//  * where the hierarchy allows it (every fine bank one coarse node, small
//    upper levels) the solve runs in the resident form: one block per
//    first-level coarse bank keeps its vertices' CG vectors in registers and
//    its bank inverses in shared memory, two grid or cluster barriers per
//    iteration, and BF16-stored inverses are applied with mma.sync (FP32
//    accumulation).
#include <cooperative_groups.h>
#include <cuda/atomic>

#include "grid_barrier.cuh"
#include "mas_cg.cuh"

namespace silkb {

namespace {

constexpr int kCgThreads = 256;
constexpr int kCgWarps = kCgThreads / 32;

__global__ void galerkin_fill_kernel(GalerkinDev g, const double* src_vals,
                                     const float* dyn) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.n_entries) return;
  double s = 0.0;
  for (int k = g.src_off[e]; k < g.src_off[e + 1]; ++k) s += src_vals[g.src[k]];
  if (g.diag_off)
    for (int k = g.diag_off[e]; k < g.diag_off[e + 1]; ++k) s += (double)dyn[g.diag[k]];
  g.vals[e] = s;
}

// Fill one 32x32 bank matrix in FP64 and invert it in place with symmetric
// pivot sweeps (no pivoting; the bank matrices are SPD principal blocks of a
// Galerkin operator, virtual slots are identity).  A zero or non-finite pivot,
// or a non-finite inverse entry, sets kFailMasPivot in *fail and leaves the
// bank's inverse zero, as batched_invert_upper rejects such a bank
// (mas_preconditioner.cu:766-830, reported as a failed factorisation at
// :854-858).
__global__ void __launch_bounds__(256) bank_invert_kernel(
    MasLevelDev lv, int fine, const int* part_off, const double* src_vals,
    const float* dyn, int* fail) {
  __shared__ double A[BANK][BANK + 1];
  __shared__ double col[BANK], row[BANK];
  int bank = blockIdx.x;
  int size = fine ? part_off[bank + 1] - part_off[bank] : BANK;
  int base_v = fine ? part_off[bank] : 0;
  for (int e = threadIdx.x; e < BANK * BANK; e += blockDim.x) {
    int i = e / BANK, j = e % BANK;
    int idx = upper_index(BANK, i, j);
    int src = lv.fill_src[(size_t)bank * kPacked + idx];
    double v = src >= 0 ? src_vals[src] : 0.0;
    if (i == j) {
      if (fine && i < size) v += (double)dyn[base_v + i];
      if (v == 0.0) v = 1.0;  // pad_zero_diagonal
    }
    A[i][j] = v;
  }
  __syncthreads();
  for (int k = 0; k < BANK; ++k) {
    if (threadIdx.x < BANK) {
      col[threadIdx.x] = A[threadIdx.x][k];
      row[threadIdx.x] = A[k][threadIdx.x];
    }
    __syncthreads();
    double p = col[k];
    if (!isfinite(p) || p == 0.0) {  // uniform: every thread reads the same pivot
      if (threadIdx.x == 0 && fail) atomicOr(fail, kFailMasPivot);
      for (int idx = threadIdx.x; idx < kPacked; idx += blockDim.x) {
        if (lv.M) lv.M[(size_t)bank * kPacked + idx] = 0.0f;
        if (lv.Mb) lv.Mb[(size_t)bank * kPacked + idx] = __float2bfloat16_rn(0.0f);
      }
      return;
    }
    double inv = 1.0 / p;
    for (int e = threadIdx.x; e < BANK * BANK; e += blockDim.x) {
      int i = e / BANK, j = e % BANK;
      double v;
      if (i == k && j == k) v = inv;
      else if (i == k) v = row[j] * inv;
      else if (j == k) v = -col[i] * inv;
      else v = A[i][j] - col[i] * row[j] * inv;
      A[i][j] = v;
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kPacked; idx += blockDim.x) {
    // Invert the packed-upper index.
    int i = 0, rem = idx;
    while (rem >= BANK - i) {
      rem -= BANK - i;
      ++i;
    }
    int j = i + rem;
    double v = A[i][j];
    if (!isfinite((float)v)) {
      if (fail) atomicOr(fail, kFailMasPivot);
      v = 0.0;
    }
    if (lv.M) lv.M[(size_t)bank * kPacked + idx] = (float)v;
    if (lv.Mb) lv.Mb[(size_t)bank * kPacked + idx] = __float2bfloat16_rn((float)v);
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One lane's share of a fixed-order sum over per-block partials (4 doubles
// per block, slot `slot`): the values of blocks lane, lane + 32, ... added in
// that order, as the strided loop would, with the first kLoads of them loaded
// from L2 before the first add (one round trip instead of one per value).  An
// absent value adds +0.0, which leaves a sum started at +0.0 unchanged bit
// for bit (such a sum is never -0.0).
template <int kLoads>
__device__ __forceinline__ double lane_partials(const double* partials, int slot, int nblocks,
                                                int lane) {
  double v[kLoads];
#pragma unroll
  for (int k = 0; k < kLoads; ++k) {
    const int b = lane + 32 * k;
    v[k] = b < nblocks ? __ldcg(partials + 4 * b + slot) : 0.0;
  }
  double a = 0.0;
#pragma unroll
  for (int k = 0; k < kLoads; ++k) a += v[k];
  for (int b = lane + 32 * kLoads; b < nblocks; b += 32) a += __ldcg(partials + 4 * b + slot);
  return a;
}
// Loads in flight per lane for the resident form's totals: its cooperative
// grid has one block per SM (148 on B200), at most 160 blocks in one round.
constexpr int kResPartialLoads = 5;

// Block-level sum of per-thread doubles into out[k] (thread 0 writes).
template <int N>
__device__ void block_sum(double (&v)[N], double* out) {
  __shared__ double sh[N][kCgWarps];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double a = warp_sum_d(v[k]);
    if (lane == 0) sh[k][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double a = lane < kCgWarps ? sh[k][lane] : 0.0;
      a = warp_sum_d(a);
      if (lane == 0) out[k] = a;
    }
  }
  __syncthreads();
}

// Every block sums slot `slot` of the per-block partials in the same order.
__device__ double grid_total(const double* partials, int slot, int nblocks) {
  __shared__ double s_tot;
  if (threadIdx.x < 32) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) a += partials[4 * b + slot];
    a = warp_sum_d(a);
    if (threadIdx.x == 0) s_tot = a;
  }
  __syncthreads();
  double t = s_tot;
  __syncthreads();
  return t;
}

// Stage a packed bank inverse into shared memory as FP32.
__device__ __forceinline__ void stage_bank(const MasLevelDev& lv, int bf16,
                                           int bank, float* sm, int lane) {
  if (bf16) {
    const __nv_bfloat16* src = lv.Mb + (size_t)bank * kPacked;
    for (int k = lane; k < kPacked; k += 32) sm[k] = __bfloat162float(src[k]);
  } else {
    const float4* src = reinterpret_cast<const float4*>(lv.M + (size_t)bank * kPacked);
    for (int k = lane; k < kPacked / 4; k += 32) {
      float4 q = src[k];
      sm[4 * k] = q.x;
      sm[4 * k + 1] = q.y;
      sm[4 * k + 2] = q.z;
      sm[4 * k + 3] = q.w;
    }
  }
  __syncwarp();
}

// z (lane row) = M r over the 32 slots of a bank, 3 channels.
__device__ __forceinline__ float3 bank_apply(const float* sm, float3 r,
                                             int lane) {
  float zx = 0.f, zy = 0.f, zz = 0.f;
#pragma unroll 8
  for (int k = 0; k < BANK; ++k) {
    float m = sm[upper_index(BANK, lane, k)];
    zx += m * __shfl_sync(0xffffffffu, r.x, k);
    zy += m * __shfl_sync(0xffffffffu, r.y, k);
    zz += m * __shfl_sync(0xffffffffu, r.z, k);
  }
  return make_float3(zx, zy, zz);
}

// bank_apply with the bank's residuals read from shared memory (rs[k]: slot
// k of the bank, zero where the slot is empty) as one broadcast per column
// instead of three shuffles: the same products summed in the same order.
// Used where 32 warps apply their banks at once (the shuffles' throughput,
// not their latency, is then the limit).
__device__ __forceinline__ float3 bank_apply_smem(const float* sm, const float4* rs,
                                                  int lane) {
  float zx = 0.f, zy = 0.f, zz = 0.f;
#pragma unroll 8
  for (int k = 0; k < BANK; ++k) {
    float m = sm[upper_index(BANK, lane, k)];
    float4 rk = rs[k];
    zx += m * rk.x;
    zy += m * rk.y;
    zz += m * rk.z;
  }
  return make_float3(zx, zy, zz);
}

// Restriction of the bank residual onto its connected components.
__device__ __forceinline__ void bank_restrict(const MasLevelDev& lv, int bank,
                                              float3 r, int lane) {
  if (!lv.rout) return;
  int n = lv.ncco[bank];
  int base = lv.cco_base[bank];
  int mine = lv.slot_cco[(size_t)bank * BANK + lane];
  for (int c = 0; c < n; ++c) {
    float sx = warp_sum(mine == c ? r.x : 0.f);
    float sy = warp_sum(mine == c ? r.y : 0.f);
    float sz = warp_sum(mine == c ? r.z : 0.f);
    if (lane == 0) lv.rout[base + c] = make_float4(sx, sy, sz, 0.f);
  }
}

// y = (Ldiag + dyn) v + L_off v; returns this thread's v . y contribution.
// mode 0: y = A v (store to out), mode 1: out = b - A v.
__device__ double spmv_phase(const CgArgs& a, const float4* v, float4* out,
                             int mode) {
  int lane = threadIdx.x & 31;
  int gwarp = blockIdx.x * kCgWarps + (threadIdx.x >> 5);
  int nwarps = gridDim.x * kCgWarps;
  double acc = 0.0;
  for (int s = gwarp; s < a.nslices; s += nwarps) {
    int row = 32 * s + lane;
    int base = a.sl_ptr[s], width = a.sl_w[s];
    if (row < a.nv) {
      float4 vi = v[row];
      float d = a.Ldiag[row] + a.dyn[row];
      float yx = d * vi.x, yy = d * vi.y, yz = d * vi.z;
#pragma unroll 4
      for (int k = 0; k < width; ++k) {
        int2 e = a.ent[base + k * 32 + lane];
        float val = __int_as_float(e.y);
        float4 vj = v[e.x];
        yx += val * vj.x;
        yy += val * vj.y;
        yz += val * vj.z;
      }
      if (mode == 0) {
        out[row] = make_float4(yx, yy, yz, 0.f);
        acc += (double)vi.x * yx + (double)vi.y * yy + (double)vi.z * yz;
      } else {
        float4 bb = a.b[row];
        out[row] = make_float4(bb.x - yx, bb.y - yy, bb.z - yz, 0.f);
      }
    }
  }
  return acc;
}

// Fine level: optional x/r update, z0 = M0 r, restriction to coarse space 0.
__device__ void fine_phase(const CgArgs& a, float alpha, bool update,
                           float* sm_all, double& rz, double& rr) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int gwarp = blockIdx.x * kCgWarps + warp;
  int nwarps = gridDim.x * kCgWarps;
  float* sm = sm_all + warp * kPacked;
  for (int bank = gwarp; bank < a.nbank0; bank += nwarps) {
    int base = a.part_off[bank];
    int size = a.part_off[bank + 1] - base;
    stage_bank(a.fine, a.bf16, bank, sm, lane);
    float3 rv = make_float3(0.f, 0.f, 0.f);
    int vtx = base + lane;
    if (lane < size) {
      float4 r4 = a.r[vtx];
      if (update) {
        float4 p4 = a.p[vtx], ap4 = a.Ap[vtx], x4 = a.x[vtx];
        x4.x = alpha * p4.x + x4.x;
        x4.y = alpha * p4.y + x4.y;
        x4.z = alpha * p4.z + x4.z;
        r4.x = -alpha * ap4.x + r4.x;
        r4.y = -alpha * ap4.y + r4.y;
        r4.z = -alpha * ap4.z + r4.z;
        a.x[vtx] = x4;
        a.r[vtx] = r4;
      }
      rv = make_float3(r4.x, r4.y, r4.z);
    }
    float3 z = bank_apply(sm, rv, lane);
    if (lane < size) {
      a.z0[vtx] = make_float4(z.x, z.y, z.z, 0.f);
      rz += (double)rv.x * z.x + (double)rv.y * z.y + (double)rv.z * z.z;
      rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z;
    }
    bank_restrict(a.fine, bank, rv, lane);
    __syncwarp();
  }
}

// All coarse levels, by block 0 only (they are small: ~V/1000 banks).
__device__ double coarse_phase(const CgArgs& a, float* sm_all) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* sm = sm_all + warp * kPacked;
  double rz = 0.0;
  for (int l = 0; l < a.levels; ++l) {
    const MasLevelDev& lv = a.coarse[l];
    for (int bank = warp; bank < lv.nbank; bank += kCgWarps) {
      int node = bank * BANK + lane;
      bool valid = node < lv.nnode;
      float3 rv = make_float3(0.f, 0.f, 0.f);
      if (valid) {
        float4 q = lv.rin[node];
        rv = make_float3(q.x, q.y, q.z);
      }
      stage_bank(lv, a.bf16, bank, sm, lane);
      float3 z = bank_apply(sm, rv, lane);
      if (valid) {
        lv.zout[node] = make_float4(z.x, z.y, z.z, 0.f);
        rz += (double)rv.x * z.x + (double)rv.y * z.y + (double)rv.z * z.z;
      }
      bank_restrict(lv, bank, rv, lane);
      __syncwarp();
    }
    __syncthreads();
  }
  return rz;
}

__device__ void prolong_phase(const CgArgs& a, float beta) {
  int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nv; v += stride) {
    float4 z = a.z0[v];
    if (a.levels > 0) {
      int4 cm = a.cmap[v];
      int ids[4] = {cm.x, cm.y, cm.z, cm.w};
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        if (l >= a.levels) break;
        float4 q = a.coarse[l].zout[ids[l]];
        z.x += q.x;
        z.y += q.y;
        z.z += q.z;
      }
    }
    float4 p = a.p[v];
    // beta == 0 (first iteration or guarded ratio) sets p = z exactly.
    a.p[v] = beta == 0.0f ? make_float4(z.x, z.y, z.z, 0.f)
                          : make_float4(z.x + beta * p.x, z.y + beta * p.y,
                                        z.z + beta * p.z, 0.f);
  }
}

// Hardware barrier of a thread-block cluster: used when the whole solve runs
// in one cluster (small and medium systems), where it replaces the global
// memory barrier that dominates the CG iteration time of such systems.
struct ClusterBarrier {
  __device__ bool sync() {
    cooperative_groups::this_cluster().sync();
    return true;
  }
};

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Phase stamps of block 0 (slots: 0 prolongation done, 1 its barrier passed,
// 2 SpMV done, 3 barrier, 4 fine level done, 5 barrier, 6 coarse levels
// done, 7 barrier).
struct CgTrace {
  long long* t;
  __device__ CgTrace(long long* p, int form)
      : t(blockIdx.x == 0 && threadIdx.x == 0 ? p : nullptr) {
    if (t) {
      t[0] = global_ns();
      t[1] = clock64();
      t[5] = form;
    }
  }
  __device__ __forceinline__ void stamp(int iter, int slot) {
    if (t && iter >= 0 && iter < kCgTraceIters) {
      long long c = clock64();
      for (int k = slot; k < kCgTraceSlots; ++k) t[8 + iter * kCgTraceSlots + k] = c;
    }
  }
  __device__ void finish(int iters) {
    if (!t) return;
    t[2] = global_ns();
    t[3] = clock64();
    t[4] = iters < kCgTraceIters ? iters : kCgTraceIters;
  }
};

// Weight w of the start x + w (x_alt - x) whose residual r + w (r_alt - r)
// has the smallest norm: w = <r, r - r_alt> / |r - r_alt|^2.  Used only when
// it lowers |r|^2 by at least 1 % (otherwise w = 0, the plain start), so the
// blend never raises the residual; w = 1 is the alternative start itself.
__device__ __forceinline__ double blend_weight(double rr, double r_ra, double rara) {
  double den = rr - 2.0 * r_ra + rara;
  if (!(den > 0.0) || !(rr > 0.0)) return 0.0;
  double num = rr - r_ra;
  if (num <= 0.0 || num * num < 1e-2 * den * rr) return 0.0;
  double w = num / den;
  return isfinite(w) ? w : 0.0;
}

__device__ __forceinline__ void mark_fail(const CgArgs& a) {
  if (threadIdx.x == 0 && a.fail) atomicOr(a.fail, kFailBarrier);
}

template <class Barrier>
__device__ __forceinline__ void cg_body(const CgArgs& a, Barrier& bar, float* sm_all) {
  if (a.skip && *a.skip) return;  // the ADMM solve already ended (every block alike)
  double* part = a.partials + 4 * blockIdx.x;
  CgTrace tr(a.trace, 0);
  // r = b - A x.
  spmv_phase(a, a.x, a.r, 1);
  if (!bar.sync()) return mark_fail(a);
  // Alternative start (see CgArgs::x_alt): its residual goes to Ap.
  double rr_plain0 = -1.0;
  if (a.x_alt) {
    spmv_phase(a, a.x_alt, a.Ap, 1);
    if (!bar.sync()) return mark_fail(a);
    {
      double v[3] = {0.0, 0.0, 0.0};
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nv; i += gridDim.x * blockDim.x) {
        float4 q = a.r[i], w = a.Ap[i];
        v[0] += (double)q.x * q.x + (double)q.y * q.y + (double)q.z * q.z;
        v[1] += (double)q.x * w.x + (double)q.y * w.y + (double)q.z * w.z;
        v[2] += (double)w.x * w.x + (double)w.y * w.y + (double)w.z * w.z;
      }
      block_sum<3>(v, part);
    }
    if (!bar.sync()) return mark_fail(a);
    const double rr_plain = grid_total(a.partials, 0, gridDim.x);
    const double r_pa = grid_total(a.partials, 1, gridDim.x);
    const double rr_alt = grid_total(a.partials, 2, gridDim.x);
    if (!bar.sync()) return mark_fail(a);
    rr_plain0 = rr_plain;
    const float w = (float)blend_weight(rr_plain, r_pa, rr_alt);
    if (w > 0.0f) {
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nv; i += gridDim.x * blockDim.x) {
        float4 x0 = a.x[i], xa = a.x_alt[i], r0 = a.r[i], ra = a.Ap[i];
        a.x[i] = make_float4(x0.x + w * (xa.x - x0.x), x0.y + w * (xa.y - x0.y),
                             x0.z + w * (xa.z - x0.z), 0.f);
        a.r[i] = make_float4(r0.x + w * (ra.x - r0.x), r0.y + w * (ra.y - r0.y),
                             r0.z + w * (ra.z - r0.z), 0.f);
      }
      if (blockIdx.x == 0 && threadIdx.x == 0 && a.stats) atomicAdd(a.stats + a.alt_stat, 1);
      if (!bar.sync()) return mark_fail(a);
    }
  }
  {
    double v[2] = {0.0, 0.0};
    fine_phase(a, 0.f, false, sm_all, v[0], v[1]);
    block_sum<2>(v, part);
  }
  if (!bar.sync()) return mark_fail(a);
  if (blockIdx.x == 0) {
    double v[1] = {coarse_phase(a, sm_all)};
    block_sum<1>(v, a.coarse_partial);
  }
  if (!bar.sync()) return mark_fail(a);
  double rz = grid_total(a.partials, 0, gridDim.x) + *a.coarse_partial;
  double rr = grid_total(a.partials, 1, gridDim.x);
  if (!isfinite(rz)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.result[0] = 0;
      a.result[1] = kCgInvalidInitialResidual;
      *a.result_rr = (float)rr;
    }
    return;
  }
  const double rr0 = rr_plain0 >= 0.0 ? rr_plain0 : rr;
  const double abs2 = (double)a.abs_tol * a.abs_tol;
  const float rel_tol = a.rel_tol_dev ? *a.rel_tol_dev : a.rel_tol;
  const double rel2 = (double)rel_tol * rel_tol;
  double beta = 0.0;
  int iter = 0;
  int status = kCgMaxIter;
  while (true) {
    prolong_phase(a, (float)beta);
    tr.stamp(iter, 0);
    if (!bar.sync()) return mark_fail(a);
    tr.stamp(iter, 1);
    {
      double v[1] = {spmv_phase(a, a.p, a.Ap, 0)};
      block_sum<1>(v, part + 2);
    }
    tr.stamp(iter, 2);
    if (!bar.sync()) return mark_fail(a);
    tr.stamp(iter, 3);
    double pAp = grid_total(a.partials, 2, gridDim.x);
    double alpha = fabs(pAp) < 1e-20 ? 0.0 : rz / pAp;
    {
      double v[2] = {0.0, 0.0};
      fine_phase(a, (float)alpha, true, sm_all, v[0], v[1]);
      block_sum<2>(v, part);
    }
    tr.stamp(iter, 4);
    if (!bar.sync()) return mark_fail(a);
    tr.stamp(iter, 5);
    if (blockIdx.x == 0) {
      double v[1] = {coarse_phase(a, sm_all)};
      block_sum<1>(v, a.coarse_partial);
    }
    tr.stamp(iter, 6);
    if (!bar.sync()) return mark_fail(a);
    tr.stamp(iter, 7);
    double rz_old = rz;
    rz = grid_total(a.partials, 0, gridDim.x) + *a.coarse_partial;
    rr = grid_total(a.partials, 1, gridDim.x);
    ++iter;
    bool stop = false;
    if (iter >= a.max_iter) {
      status = kCgMaxIter;
      stop = true;
    } else if (rr <= abs2) {
      status = kCgAbsTol;
      stop = true;
    } else if (rr <= rel2 * rr0) {
      status = kCgRelTol;
      stop = true;
    }
    beta = fabs(rz_old) < 1e-20 ? 0.0 : rz / rz_old;
    if (stop) break;
  }
  tr.finish(iter);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.result[0] = iter;
    a.result[1] = status;
    *a.result_rr = (float)rr;
    if (a.stats) {
      atomicAdd(a.stats, iter);
      atomicAdd(a.stats + 1, 1);
      if (a.first_solve) atomicAdd(a.stats + 2, iter);
    }
  }
}

__global__ void __launch_bounds__(kCgThreads) cg_kernel(CgArgs a) {
  extern __shared__ float sm_all[];
  GridBarrier bar{a.barrier, a.barrier + 1, a.barrier + 2, gridDim.x};
  if (a.barrier_spin_limit > 0) bar.limit = a.barrier_spin_limit;
  if (a.withhold_block >= 0) bar.withhold = (unsigned)a.withhold_block;
  cg_body(a, bar, sm_all);
}

__global__ void __launch_bounds__(kCgThreads) cg_kernel_cluster(CgArgs a) {
  extern __shared__ float sm_all[];
  ClusterBarrier bar;
  cg_body(a, bar, sm_all);
}

// ---------------------------------------------------------------------------
// Resident PCG: block k owns first-level coarse bank k, i.e. the fine banks
// 32k .. 32k+31, with one thread per fine-bank slot (warp w = fine bank
// 32k+w, lane = slot).  Every vertex's x, r, p, Ap and its MAS output stay
// in registers for the whole solve; the block's fine and first-level bank
// inverses and the (few) banks of all higher levels are staged in shared
// memory once per solve.  What crosses blocks: each vertex's two-level z
// (fine + first coarse level) for the blocks whose halo holds it, the
// per-block partial sums and the residual restricted to the second coarse
// level, which every block then solves redundantly.  Each block computes p
// at its halo vertices itself with the owner's operations (bit-identical),
// so p needs no barrier of its own (when a block's halo overflows its
// shared-memory slots, p is published through the grid as well):
//   A  totals, coarse levels >= 2, p = z + beta p (own and halo)   | block barrier
//   B  Ap = A p (bank-sliced ELL in a bank-group-conflict-free     |
//      order, vertex and halo slots in shared memory), p.Ap partial | barrier
//   C  alpha, x/r update, fine and first-level MAS, restriction,   | barrier
//      two-level z published, r.z and r.r partials
// The arithmetic of each vector entry is that of cg_kernel except the order
// of the FP64 block sums, of the off-diagonal terms of a row (the scheduled
// order) and of the upper-level bank solves (columns split over warps).
// ---------------------------------------------------------------------------
constexpr int kResWarps = kResThreads / 32;
static_assert(kResCoarseBanks <= kResWarps, "one warp per upper coarse bank");

// A bank slot of shared memory holds either the packed FP32 inverse (528
// floats) or, for BF16 storage, the inverse as mma.m16n8k16 A fragments:
// 4 tiles (2 row x 2 column halves) x 32 lanes x 8 bf16 = 2048 bytes.
struct ResShared {
  float Mf[kResWarps][kPacked];
  float M1[kPacked];
  float Mc[kResCoarseBanks][kPacked];
  float4 pl[kResThreads + kResHalo];  // the block's slots, then its halo
  int4 hcm[kResHalo];                 // coarse nodes of the halo vertices (cmap)
  float4 r1[32];
  float4 z1[32];
  float4 rc[kResCoarseBanks * BANK];
  float4 zc[kResCoarseBanks * BANK];
  __nv_bfloat16 rb[kResWarps][8][BANK];  // BF16 apply: residual as B operand (rows 3..7 zero)
  float4 zs[kResWarps][BANK];             // BF16 apply: accumulator rows back to slots
  double red[kResWarps][3];
  double tot[3];
  unsigned tmem_base;  // tensor-memory address of the block's row store
};
static_assert(offsetof(ResShared, M1) % 16 == 0 && offsetof(ResShared, Mc) % 16 == 0 &&
                  (kPacked * sizeof(float)) % 16 == 0,
              "bank slots hold 16-byte fragments");

// Stage a bank inverse stored as packed BF16 into A-fragment order: lane
// (g = lane / 4, t = lane % 4) of tile (mt, kt) holds rows 16 mt + g (+8) and
// columns 16 kt + 2t (+1, +8, +9), the m16n8k16 row-major A layout.
__device__ __forceinline__ void stage_bank_frag(const MasLevelDev& lv, int bank, float* slot,
                                                int lane) {
  const __nv_bfloat16* src = lv.Mb + (size_t)bank * kPacked;
  uint4* dst = reinterpret_cast<uint4*>(slot);
  const int g = lane >> 2, t = lane & 3;
  auto pair = [&](int i, int j) -> unsigned {
    unsigned lo = __bfloat16_as_ushort(src[upper_index(BANK, i, j)]);
    unsigned hi = __bfloat16_as_ushort(src[upper_index(BANK, i, j + 1)]);
    return lo | (hi << 16);
  };
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const int r0 = 16 * mt + g, c0 = 16 * kt + 2 * t;
      uint4 q;
      q.x = pair(r0, c0);
      q.y = pair(r0 + 8, c0);
      q.z = pair(r0, c0 + 8);
      q.w = pair(r0 + 8, c0 + 8);
      dst[(mt * 2 + kt) * 32 + lane] = q;
    }
  __syncwarp();
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint4& a, unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// z (lane slot) = M r on the tensor cores: Z (32 x 8) = M (32 x 32) R (32 x 8),
// R holding the three channels of r in BF16 and zero columns 3..7, FP32
// accumulation; four m16n8k16 products per bank.
__device__ __forceinline__ float3 bank_apply_mma(const float* slot, float3 r, int lane,
                                                 __nv_bfloat16 (*rb)[BANK], float4* zs) {
  rb[0][lane] = __float2bfloat16_rn(r.x);
  rb[1][lane] = __float2bfloat16_rn(r.y);
  rb[2][lane] = __float2bfloat16_rn(r.z);
  __syncwarp();
  const int g = lane >> 2, t = lane & 3;
  const unsigned* rw = reinterpret_cast<const unsigned*>(&rb[g][0]);
  unsigned b[2][2];
#pragma unroll
  for (int kt = 0; kt < 2; ++kt) {
    b[kt][0] = rw[kt * 8 + t];
    b[kt][1] = rw[kt * 8 + 4 + t];
  }
  const uint4* frag = reinterpret_cast<const uint4*>(slot);
  float c[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) mma_bf16(c[mt], frag[(mt * 2 + kt) * 32 + lane], b[kt][0], b[kt][1]);
  if (t < 2) {
    float* z = reinterpret_cast<float*>(zs);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int row = 16 * mt + g;
      *reinterpret_cast<float2*>(z + 4 * row + 2 * t) = make_float2(c[mt][0], c[mt][1]);
      *reinterpret_cast<float2*>(z + 4 * (row + 8) + 2 * t) = make_float2(c[mt][2], c[mt][3]);
    }
  }
  __syncwarp();
  float4 q = zs[lane];
  __syncwarp();
  return make_float3(q.x, q.y, q.z);
}

// Block sums of up to three doubles per thread, in a fixed order; thread 0
// of the block stores them to out (global) when out is not null.  The sums
// are left in s.tot.  kFinalSync = false skips the closing block barrier
// where the caller's next step is a grid or cluster barrier anyway (which
// also orders the next reuse of s.red and s.tot).
template <int N, bool kFinalSync = true>
__device__ void res_block_sum(const double (&v)[N], ResShared& s, double* out) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double a = warp_sum_d(v[k]);
    if (lane == 0) s.red[warp][k] = a;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double a = warp_sum_d(s.red[lane][k]);
      if (lane == 0) {
        s.tot[k] = a;
        if (out) out[k] = a;
      }
    }
  }
  if (kFinalSync) __syncthreads();
}

// Sum of slot `slot` of every block's partials, the same in every block.
__device__ double res_total(const double* partials, int slot, int nblocks, ResShared& s) {
  if (threadIdx.x < 32) {
    double a = lane_partials<kResPartialLoads>(partials, slot, nblocks, threadIdx.x);
    a = warp_sum_d(a);
    if (threadIdx.x == 0) s.tot[slot] = a;
  }
  __syncthreads();
  double t = s.tot[slot];
  __syncthreads();
  return t;
}

__device__ __forceinline__ float4 ldcg4(const float4* p) { return __ldcg(p); }

// Tensor memory (sm_100a) as a per-CTA store for the SpMV rows.  A warp
// reaches the 32 lanes 32 (w % 4) .. 32 (w % 4) + 31 of it; lane = row
// (bank slot), two 32-bit columns per row entry (column index, value).
// Every tcgen05 instruction here is warp-collective and runs in warp-uniform
// control flow.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tmem_alloc(unsigned* dst, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
               ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// Store 16 columns of this thread's lane, then wait for the warp's stores.
__device__ __forceinline__ void tmem_st16_wait(unsigned taddr, const unsigned (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};\n"
      "tcgen05.wait::st.sync.aligned;\n"
      ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]),
      "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]),
      "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
// Load 16 columns of this thread's lane; the wait is in the same statement,
// so no use of the outputs can be scheduled before it.
__device__ __forceinline__ void tmem_ld16_wait(unsigned taddr, unsigned (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}

// Off-diagonal row sum of this thread's vertex plus the diagonal term.
__device__ __forceinline__ float3 res_row(const CgArgs& a, const ResShared& s,
                                          const float4* ex, int rptr, int rw,
                                          int lane, float d, float3 pv) {
  float yx = d * pv.x, yy = d * pv.y, yz = d * pv.z;
  const int2* e = a.rent + rptr + lane;
#pragma unroll 4
  for (int j = 0; j < rw; ++j) {
    int2 q = e[j * BANK];
    float val = __int_as_float(q.y);
    float4 pj = q.x < 0 ? s.pl[-1 - q.x] : ldcg4(ex + q.x);
    yx = fmaf(val, pj.x, yx);
    yy = fmaf(val, pj.y, yy);
    yz = fmaf(val, pj.z, yz);
  }
  return make_float3(yx, yy, yz);
}

// res_row with the row entries read from tensor memory, eight per load (the
// entries of res_row in the same order, so the same sums).
__device__ __forceinline__ float3 res_row_tmem(const ResShared& s, const float4* ex,
                                               unsigned taddr, int rw, float d, float3 pv) {
  float yx = d * pv.x, yy = d * pv.y, yz = d * pv.z;
  for (int j0 = 0; j0 < rw; j0 += 8) {
    unsigned e[16];
    tmem_ld16_wait(taddr + 2 * j0, e);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (j0 + k < rw) {
        const int col = (int)e[2 * k];
        const float val = __uint_as_float(e[2 * k + 1]);
        const float4 pj = col < 0 ? s.pl[-1 - col] : ldcg4(ex + col);
        yx = fmaf(val, pj.x, yx);
        yy = fmaf(val, pj.y, yy);
        yz = fmaf(val, pj.z, yz);
      }
    }
  }
  return make_float3(yx, yy, yz);
}

template <class Barrier>
__device__ void res_body(const CgArgs& a, Barrier& bar, ResShared& s) {
  if (a.skip && *a.skip) return;  // the ADMM solve already ended (every block alike)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = blockIdx.x;
  const int nblocks = gridDim.x;
  const int fb = k * BANK + warp;
  const bool bank_ok = fb < a.nbank0;
  const bool has1 = a.levels > 0;
  CgTrace tr(a.trace, 1);
  int iter = -1;  // -1 while setting up (not traced)
  double* part = a.partials + 4 * k;
  // Row store in tensor memory (allocated after the staging below): every
  // warp's accesses complete before warp 0 frees it, on every way out.
  unsigned taddr = 0;
  bool tm = false;
  auto tm_release = [&]() {
    if (a.tm_cols <= 0) return;
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
      tmem_fence_after();
      tmem_dealloc(s.tmem_base, (unsigned)a.tm_cols);
    }
  };
  auto fail = [&]() {
    tm_release();
    if (tid == 0 && a.fail) atomicOr(a.fail, kFailBarrier);
  };

  // ---- one-time staging ----------------------------------------------------
  // BF16 storage: inverses staged as tensor-core fragments and applied with
  // mma.sync; FP32 storage: packed FP32 and the SIMT apply.
  const bool tc = a.bf16 != 0;
  auto stage = [&](const MasLevelDev& lv, int bank, float* slot) {
    if (tc)
      stage_bank_frag(lv, bank, slot, lane);
    else
      stage_bank(lv, 0, bank, slot, lane);
  };
  auto apply = [&](const float* slot, float3 r) {
    return tc ? bank_apply_mma(slot, r, lane, s.rb[warp], s.zs[warp]) : bank_apply(slot, r, lane);
  };
  for (int i = lane; i < 5 * BANK; i += 32) s.rb[warp][3 + i / BANK][i % BANK] = __float2bfloat16_rn(0.f);
  int vbase = 0, vsize = 0, rptr = 0, rw = 0;
  if (bank_ok) {
    vbase = a.part_off[fb];
    vsize = a.part_off[fb + 1] - vbase;
    rptr = a.rb_ptr[fb];
    rw = a.rb_w[fb];
    stage(a.fine, fb, s.Mf[warp]);
  }
  const bool own = lane < vsize;
  const int v = vbase + lane;
  if (has1 && warp == 0) stage(a.coarse[0], k, s.M1);
  // Warp w keeps its bank's rows in lanes 32 (w % 4).. of the row store and
  // columns 2 tm_rw (w / 4) .., entries past the bank's width padded with
  // (own slot, 0) and never read.
  if (a.tm_cols > 0) {
    tm = (kResWarps / 4) * 2 * a.tm_rw <= a.tm_cols && rw <= a.tm_rw;
    if (warp == 0) tmem_alloc(&s.tmem_base, (unsigned)a.tm_cols);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    taddr = s.tmem_base + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)((warp >> 2) * 2 * a.tm_rw);
    if (tm) {
      const int2* erow = a.rent + rptr + lane;
      for (int j0 = 0; j0 < rw; j0 += 8) {
        unsigned e[16];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int2 qe = j0 + q < rw ? erow[(j0 + q) * BANK] : make_int2(-1 - tid, 0);
          e[2 * q] = (unsigned)qe.x;
          e[2 * q + 1] = (unsigned)qe.y;
        }
        tmem_st16_wait(taddr + 2 * j0, e);
      }
    }
  }

  // First-level restriction plan of this block's coarse bank (warp 0).
  int l1_ncco = 0, l1_base = 0, l1_mine = -1;
  if (has1 && warp == 0 && a.levels > 1) {
    l1_ncco = a.coarse[0].ncco[k];
    l1_base = a.coarse[0].cco_base[k];
    l1_mine = a.coarse[0].slot_cco[(size_t)k * BANK + lane];
  }
  {
    int cb = 0;
    for (int l = 1; l < a.levels; ++l) {
      for (int j = warp; j < a.coarse[l].nbank; j += kResWarps)
        stage(a.coarse[l], j, s.Mc[cb + j]);
      cb += a.coarse[l].nbank;
    }
    for (int i = tid; i < kResCoarseBanks * BANK; i += kResThreads)
      s.rc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  float d = 0.f;
  float3 x = make_float3(0.f, 0.f, 0.f), b = x;
  int cm[4] = {-1, -1, -1, -1};
  if (own) {
    d = a.Ldiag[v] + a.dyn[v];
    float4 x4 = a.x[v], b4 = a.b[v];
    x = make_float3(x4.x, x4.y, x4.z);
    b = make_float3(b4.x, b4.y, b4.z);
    if (has1) {
      int4 c = a.cmap[v];
      cm[0] = c.x;
      cm[1] = c.y;
      cm[2] = c.z;
      cm[3] = c.w;
    }
  }
  auto row = [&](const float4* ex, float3 pv) {
    return tm ? res_row_tmem(s, ex, taddr, rw, d, pv) : res_row(a, s, ex, rptr, rw, lane, d, pv);
  };
  // Halo: thread i < nhalo gathers halo vertex i of the block into slot
  // kResThreads + i before each product (one round trip, all loads in flight).
  int hcol = -1;
  if (a.halo_off) {
    const int h0 = a.halo_off[k], nh = a.halo_off[k + 1] - h0;
    if (tid < nh) hcol = a.halo_col[h0 + tid];
  }
  // With every off-block column in the halo, the block computes p at its
  // halo vertices itself (owner's two-level z, published before the barrier
  // that ends phase C, plus the upper levels every block holds), so p needs
  // no publication barrier.
  const bool halo_p = a.halo_full != 0;
  if (halo_p && hcol >= 0 && has1) s.hcm[tid] = a.cmap[hcol];
  auto gather_halo = [&](const float4* ex) {
    if (hcol >= 0) s.pl[kResThreads + tid] = ldcg4(ex + hcol);
    __syncthreads();
  };
  // Publish x for r = b - A x.
  s.pl[tid] = make_float4(x.x, x.y, x.z, 0.f);
  if (own) a.p[v] = make_float4(x.x, x.y, x.z, 0.f);
  if (!bar.sync()) return fail();
  gather_halo(a.p);
  float3 r;
  {
    float3 y = row(a.p, x);
    r = own ? make_float3(b.x - y.x, b.y - y.y, b.z - y.z) : make_float3(0.f, 0.f, 0.f);
  }
  // Alternative start: residual of x_alt (published through the Ap buffer),
  // both residual norms summed over the grid, the smaller start taken by
  // every block alike; the plain start's norm stays the stopping reference.
  double rr_plain0 = -1.0;
  if (a.x_alt) {
    float3 xa = make_float3(0.f, 0.f, 0.f);
    if (own) {
      float4 q = a.x_alt[v];
      xa = make_float3(q.x, q.y, q.z);
    }
    __syncthreads();
    s.pl[tid] = make_float4(xa.x, xa.y, xa.z, 0.f);
    if (own) a.Ap[v] = make_float4(xa.x, xa.y, xa.z, 0.f);
    if (!bar.sync()) return fail();
    gather_halo(a.Ap);
    float3 ra;
    {
      float3 y = row(a.Ap, xa);
      ra = own ? make_float3(b.x - y.x, b.y - y.y, b.z - y.z) : make_float3(0.f, 0.f, 0.f);
    }
    const double v3[3] = {(double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z,
                          (double)r.x * ra.x + (double)r.y * ra.y + (double)r.z * ra.z,
                          (double)ra.x * ra.x + (double)ra.y * ra.y + (double)ra.z * ra.z};
    res_block_sum<3>(v3, s, part);
    if (!bar.sync()) return fail();
    const double rr_plain = res_total(a.partials, 0, nblocks, s);
    const double r_pa = res_total(a.partials, 1, nblocks, s);
    const double rr_alt = res_total(a.partials, 2, nblocks, s);
    // Every block reads the partials before any block overwrites them in the
    // next phase.
    if (!bar.sync()) return fail();
    rr_plain0 = rr_plain;
    const float w = (float)blend_weight(rr_plain, r_pa, rr_alt);
    if (w > 0.0f) {
      x = make_float3(x.x + w * (xa.x - x.x), x.y + w * (xa.y - x.y), x.z + w * (xa.z - x.z));
      r = make_float3(r.x + w * (ra.x - r.x), r.y + w * (ra.y - r.y), r.z + w * (ra.z - r.z));
      if (k == 0 && tid == 0 && a.stats) atomicAdd(a.stats + a.alt_stat, 1);
    }
  }

  // Phase C body: fine and first-level MAS of r, restriction to level 2,
  // partials (r.z, r.r) of this block.
  float3 z0, zl, p = make_float3(0.f, 0.f, 0.f), Ap = p;
  float4 hz = make_float4(0.f, 0.f, 0.f, 0.f);  // two-level z of halo vertex tid
  auto mas_fine = [&]() {
    double rr = own ? (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z : 0.0;
    if (!bank_ok) {
      z0 = make_float3(0.f, 0.f, 0.f);
    } else if (tc) {
      z0 = apply(s.Mf[warp], r);
    } else {
      // The warp's residuals go through its own slots of pl, which nothing
      // reads between the SpMV and the next publication of p.
      s.pl[tid] = make_float4(r.x, r.y, r.z, 0.f);
      __syncwarp();
      z0 = bank_apply_smem(s.Mf[warp], s.pl + warp * BANK, lane);
    }
    if (!own) z0 = make_float3(0.f, 0.f, 0.f);
    double rz = own ? (double)r.x * z0.x + (double)r.y * z0.y + (double)r.z * z0.z : 0.0;
    if (has1) {
      float sx = warp_sum(r.x), sy = warp_sum(r.y), sz = warp_sum(r.z);
      if (lane == 0) s.r1[warp] = make_float4(sx, sy, sz, 0.f);
      tr.stamp(iter, 6);
      __syncthreads();
      if (warp == 0) {
        bool valid = k * BANK + lane < a.coarse[0].nnode;
        float4 q = s.r1[lane];
        float3 r1 = valid ? make_float3(q.x, q.y, q.z) : make_float3(0.f, 0.f, 0.f);
        float3 z1 = apply(s.M1, r1);
        if (!valid) z1 = make_float3(0.f, 0.f, 0.f);
        s.z1[lane] = make_float4(z1.x, z1.y, z1.z, 0.f);
        rz += (double)r1.x * z1.x + (double)r1.y * z1.y + (double)r1.z * z1.z;
        for (int c = 0; c < l1_ncco; ++c) {
          float qx = warp_sum(l1_mine == c ? r1.x : 0.f);
          float qy = warp_sum(l1_mine == c ? r1.y : 0.f);
          float qz = warp_sum(l1_mine == c ? r1.z : 0.f);
          if (lane == 0) a.coarse[0].rout[l1_base + c] = make_float4(qx, qy, qz, 0.f);
        }
      }
    }
    tr.stamp(iter, 7);
    const double v2[2] = {rz, rr};
    res_block_sum<2, false>(v2, s, part);
    // Two-level z of this vertex (s.z1 is complete after the block sum's
    // barrier), published for the blocks whose halo holds the vertex.
    zl = z0;
    if (own && has1) {
      float4 q = s.z1[warp];
      zl.x += q.x;
      zl.y += q.y;
      zl.z += q.z;
    }
    if (halo_p && own) a.z0[v] = make_float4(zl.x, zl.y, zl.z, 0.f);
    tr.stamp(iter, 8);
  };
  // Phase A head: totals and the redundant coarse levels >= 2.
  auto totals = [&](double& rz, double& rr) {
    // One round trip: warps 0 and 1 sum the two totals' partials while the
    // other warps load the residual restricted to the second coarse level.
    if (warp < 2) {
      const double t = warp_sum_d(lane_partials<kResPartialLoads>(a.partials, warp, nblocks, lane));
      if (lane == 0) s.tot[warp] = t;
    } else if (a.levels > 1) {
      for (int i = tid - 64; i < a.coarse[1].nnode; i += kResThreads - 64)
        s.rc[i] = ldcg4(a.coarse[0].rout + i);
    }
    __syncthreads();
    tr.stamp(iter, 10);
    rz = s.tot[0];
    rr = s.tot[1];
    if (a.levels > 1) {
      // The restriction chain first (warp sums per connected component), then
      // every upper bank applied at once, one warp per bank: the levels are
      // additive, each inverse only needs its own level's input.
      int cb = 0;
      for (int l = 1; l + 1 < a.levels; ++l) {
        const MasLevelDev& lv = a.coarse[l];
        if (warp < lv.nbank) {
          bool valid = warp * BANK + lane < lv.nnode;
          float4 q = s.rc[(cb + warp) * BANK + lane];
          float3 rl = valid ? make_float3(q.x, q.y, q.z) : make_float3(0.f, 0.f, 0.f);
          int n = lv.ncco[warp], base = lv.cco_base[warp];
          int mine = lv.slot_cco[(size_t)warp * BANK + lane];
          int next = (cb + lv.nbank) * BANK;
          for (int c = 0; c < n; ++c) {
            float qx = warp_sum(mine == c ? rl.x : 0.f);
            float qy = warp_sum(mine == c ? rl.y : 0.f);
            float qz = warp_sum(mine == c ? rl.z : 0.f);
            if (lane == 0) s.rc[next + base + c] = make_float4(qx, qy, qz, 0.f);
          }
        }
        cb += lv.nbank;
        __syncthreads();
      }
      tr.stamp(iter, 11);
      double rzc = 0.0;
      // Upper banks g = 0, 1, ... (every level >= 2, level by level).  BF16:
      // one warp per bank on the tensor cores.  FP32: a bank's columns are
      // split over `split` warps (at most 16 banks, 32 warps), each writing
      // its partial rows to zs; the bank's first warp adds them in warp
      // order, so a bank solve is a chain of 32 / split columns.
      int nup = 0;
      for (int l = 1; l < a.levels; ++l) nup += a.coarse[l].nbank;
      const int split = tc ? 1 : (nup <= kResWarps / 4 ? 4 : (nup <= kResWarps / 2 ? 2 : 1));
      const int g = warp / split, part = warp - g * split;
      int gj = -1, gnode = 0;  // bank within its level, nodes of that level
      {
        int first = 0;
        for (int l = 1; l < a.levels; ++l) {
          const MasLevelDev& lv = a.coarse[l];
          if (g >= first && g < first + lv.nbank) {
            gj = g - first;
            gnode = lv.nnode;
          }
          first += lv.nbank;
        }
      }
      const bool gvalid = gj >= 0 && gj * BANK + lane < gnode;
      if (tc) {
        if (gj >= 0) {
          const int slot = g * BANK + lane;
          float4 q = s.rc[slot];
          float3 rl = gvalid ? make_float3(q.x, q.y, q.z) : make_float3(0.f, 0.f, 0.f);
          float3 zq = apply(s.Mc[g], rl);
          if (!gvalid) zq = make_float3(0.f, 0.f, 0.f);
          s.zc[slot] = make_float4(zq.x, zq.y, zq.z, 0.f);
          rzc += (double)rl.x * zq.x + (double)rl.y * zq.y + (double)rl.z * zq.z;
        }
      } else {
        if (gj >= 0) {
          // Slots of s.rc past a level's nodes are never written (zero).
          const int cols = BANK / split, k0 = part * cols;
          const float* sm = s.Mc[g];
          const float4* rs = s.rc + g * BANK;
          float zx = 0.f, zy = 0.f, zz = 0.f;
#pragma unroll 8
          for (int kk = k0; kk < k0 + cols; ++kk) {
            float m = sm[upper_index(BANK, lane, kk)];
            float4 rk = rs[kk];
            zx += m * rk.x;
            zy += m * rk.y;
            zz += m * rk.z;
          }
          s.zs[warp][lane] = make_float4(zx, zy, zz, 0.f);
        }
        __syncthreads();
        if (gj >= 0 && part == 0) {
          float4 acc = s.zs[warp][lane];
          for (int q = 1; q < split; ++q) {
            float4 t = s.zs[warp + q][lane];
            acc.x += t.x;
            acc.y += t.y;
            acc.z += t.z;
          }
          const int slot = g * BANK + lane;
          float4 q = s.rc[slot];
          float3 rl = gvalid ? make_float3(q.x, q.y, q.z) : make_float3(0.f, 0.f, 0.f);
          float3 zq = gvalid ? make_float3(acc.x, acc.y, acc.z) : make_float3(0.f, 0.f, 0.f);
          s.zc[slot] = make_float4(zq.x, zq.y, zq.z, 0.f);
          rzc += (double)rl.x * zq.x + (double)rl.y * zq.y + (double)rl.z * zq.z;
        }
      }
      tr.stamp(iter, 12);
      const double v1[1] = {rzc};
      res_block_sum<1>(v1, s, nullptr);
      rz += s.tot[0];
    }
  };
  // Phase A tail: full preconditioned residual of a vertex from its
  // two-level z and its coarse nodes (the same operations for a vertex of
  // this block and for a halo vertex, so both give its owner's bits).
  auto upper_z = [&](float3 z, const int (&c)[4]) {
    int cb = 0;
#pragma unroll
    for (int l = 1; l < 4; ++l) {
      if (l >= a.levels) break;
      float4 q = s.zc[cb * BANK + c[l]];
      z.x += q.x;
      z.y += q.y;
      z.z += q.z;
      cb += a.coarse[l].nbank;
    }
    return z;
  };
  auto mas_total = [&]() { return own && has1 ? upper_z(zl, cm) : zl; };
  auto p_update = [&](float3 z, float3 po, float bt) {
    return bt == 0.0f ? z : make_float3(z.x + bt * po.x, z.y + bt * po.y, z.z + bt * po.z);
  };

  // Every warp has finished reading pl in the residual rows before mas_fine
  // reuses it.
  __syncthreads();
  mas_fine();
  if (!bar.sync()) return fail();
  if (halo_p && hcol >= 0) hz = ldcg4(a.z0 + hcol);
  double rz, rr;
  totals(rz, rr);
  iter = 0;
  if (!isfinite(rz)) {
    if (k == 0 && tid == 0) {
      a.result[0] = 0;
      a.result[1] = kCgInvalidInitialResidual;
      *a.result_rr = (float)rr;
    }
    tm_release();
    return;
  }
  const double rr0 = rr_plain0 >= 0.0 ? rr_plain0 : rr;
  const double abs2 = (double)a.abs_tol * a.abs_tol;
  const float rel_tol = a.rel_tol_dev ? *a.rel_tol_dev : a.rel_tol;
  const double rel2 = (double)rel_tol * rel_tol;
  double beta = 0.0;
  int status = kCgMaxIter;
  while (true) {
    // A tail: p = z + beta p, published (or, with halo_p, computed at the
    // halo vertices by this block).
    {
      const float bt = (float)beta;
      p = p_update(mas_total(), p, bt);
      if (!own) p = make_float3(0.f, 0.f, 0.f);
      s.pl[tid] = make_float4(p.x, p.y, p.z, 0.f);
      if (!halo_p && own) a.p[v] = make_float4(p.x, p.y, p.z, 0.f);
      if (halo_p && hcol >= 0) {
        float3 zh = make_float3(hz.x, hz.y, hz.z);
        if (has1) {
          int4 c4 = s.hcm[tid];
          const int c[4] = {c4.x, c4.y, c4.z, c4.w};
          zh = upper_z(zh, c);
        }
        float4 po = s.pl[kResThreads + tid];
        float3 ph = p_update(zh, make_float3(po.x, po.y, po.z), bt);
        s.pl[kResThreads + tid] = make_float4(ph.x, ph.y, ph.z, 0.f);
      }
    }
    tr.stamp(iter, 0);
    if (halo_p) {
      __syncthreads();
    } else if (!bar.sync()) {
      return fail();
    }
    tr.stamp(iter, 1);
    // B: Ap and p.Ap.
    {
      if (!halo_p) gather_halo(a.p);
      Ap = row(a.p, p);
      if (!own) Ap = make_float3(0.f, 0.f, 0.f);
      tr.stamp(iter, 2);
      const double v1[1] = {own ? (double)p.x * Ap.x + (double)p.y * Ap.y + (double)p.z * Ap.z
                                : 0.0};
      res_block_sum<1, false>(v1, s, part + 2);
    }
    tr.stamp(iter, 3);
    if (!bar.sync()) return fail();
    tr.stamp(iter, 4);
    // C: alpha, x/r update, fine + first-level MAS.
    {
      double pAp = res_total(a.partials, 2, nblocks, s);
      tr.stamp(iter, 5);
      const float alpha = (float)(fabs(pAp) < 1e-20 ? 0.0 : rz / pAp);
      x = make_float3(alpha * p.x + x.x, alpha * p.y + x.y, alpha * p.z + x.z);
      r = make_float3(-alpha * Ap.x + r.x, -alpha * Ap.y + r.y, -alpha * Ap.z + r.z);
      if (!own) r = make_float3(0.f, 0.f, 0.f);
      mas_fine();
    }
    if (!bar.sync()) return fail();
    if (halo_p && hcol >= 0) hz = ldcg4(a.z0 + hcol);
    tr.stamp(iter, 9);
    // A head: totals, coarse levels, stopping rules.
    double rz_old = rz;
    totals(rz, rr);
    tr.stamp(iter, 13);
    ++iter;
    bool stop = false;
    if (iter >= a.max_iter) {
      status = kCgMaxIter;
      stop = true;
    } else if (rr <= abs2) {
      status = kCgAbsTol;
      stop = true;
    } else if (rr <= rel2 * rr0) {
      status = kCgRelTol;
      stop = true;
    }
    beta = fabs(rz_old) < 1e-20 ? 0.0 : rz / rz_old;
    if (stop) break;
  }
  tm_release();
  if (own) a.x[v] = make_float4(x.x, x.y, x.z, 0.f);
  tr.finish(iter);
  if (k == 0 && tid == 0) {
    a.result[0] = iter;
    a.result[1] = status;
    *a.result_rr = (float)rr;
    if (a.stats) {
      atomicAdd(a.stats, iter);
      atomicAdd(a.stats + 1, 1);
      if (a.first_solve) atomicAdd(a.stats + 2, iter);
    }
  }
}

__global__ void __launch_bounds__(kResThreads, 1) cg_resident_kernel(CgArgs a) {
  extern __shared__ __align__(16) unsigned char res_smem[];
  ResShared& s = *reinterpret_cast<ResShared*>(res_smem);
  GridBarrier bar{a.barrier, a.barrier + 1, a.barrier + 2, gridDim.x};
  if (a.barrier_spin_limit > 0) bar.limit = a.barrier_spin_limit;
  if (a.withhold_block >= 0) bar.withhold = (unsigned)a.withhold_block;
  res_body(a, bar, s);
}

__global__ void __launch_bounds__(kResThreads, 1) cg_resident_cluster_kernel(CgArgs a) {
  extern __shared__ __align__(16) unsigned char res_smem[];
  ResShared& s = *reinterpret_cast<ResShared*>(res_smem);
  ClusterBarrier bar;
  res_body(a, bar, s);
}

int max_cluster_size() {
  static const int size = [] {
    size_t smem = kCgWarps * kPacked * sizeof(float);
    if (cudaFuncSetAttribute(cg_kernel_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed,
                             1) != cudaSuccess) {
      cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kCgThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 16;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&n, cg_kernel_cluster, &cfg) != cudaSuccess) {
      cudaGetLastError();
      n = 8;
    }
    return n >= 16 ? 16 : (n >= 8 ? 8 : 0);
  }();
  return size;
}


// ---------------------------------------------------------------------------
// Cluster CG with redundant coarse levels, for systems whose fine banks fit
// one thread-block cluster of at most 16 CTAs of F fine banks each (F = 8 or
// 16; the 6.4K-vertex sheet: 213 fine banks on 14 CTAs of 16).  CTA q owns
// fine banks qF .. qF+F-1, one thread per bank slot; every vector entry of
// its vertices stays in registers for the whole solve.  Compared with the
// resident form (one CTA per first-level coarse bank of 32 fine banks) the
// same system spreads over twice the SMs, and the CTAs of the cluster
// exchange through distributed shared memory instead of L2:
//  * every per-CTA partial sum (p.Ap, r.z, r.r) is stored by its CTA into
//    the shared memory of every CTA of the cluster before the cluster
//    barrier, and each CTA sums the copies in its own shared memory in CTA
//    order after it (identical totals everywhere, no global round trip);
//  * the residual restricted to the first coarse level (one node per fine
//    bank) is pushed the same way, so every CTA holds the whole first-level
//    input and computes every coarse level (restriction chain and bank
//    solves of all levels, at most kDsmCoarseBanks banks) redundantly, in
//    the same order, with identical results;
//  * p at a halo vertex is computed by the CTA itself from the owner's
//    fine-level z (stored by the owner into the CTA's shared memory before
//    the barrier) and the coarse z every CTA holds, with the owner's
//    operations.
// Per iteration: p update | CTA barrier | SpMV + p.Ap | cluster barrier |
// alpha, x/r update, fine MAS, pushes | cluster barrier | totals and coarse
// levels.  Arithmetic per vector entry as in cg_resident_kernel except the
// order of the FP64 sums and of the coarse bank solves.
// ---------------------------------------------------------------------------
constexpr int kDsmCoarseBanks = kDsmCoarseBankLimit;  // held by every CTA
constexpr int kDsmMaxCtas = 16;
constexpr int kDsmPartSlots = 8;     // 0 r.z, 1 r.r, 2 p.Ap, 3..5 alternative start

// Bank inverses in shared memory: FP32 as the full symmetric 32 x 32 matrix,
// column-major (entry (row i, column k) at k * 32 + i), so that the 32 lanes
// of a bank apply read one column in one conflict-free pass; BF16 as the
// mma.m16n8k16 A fragments (the first 2 KB of the slot).
constexpr int kDsmBankFloats = BANK * BANK;

template <int W>
struct DsmShared {
  float Mf[W][kDsmBankFloats];                // the CTA's fine bank inverses
  float Mc[kDsmCoarseBanks][kDsmBankFloats];  // every coarse bank of every level
  float4 pl[2 * 32 * W];                  // own slots, then the halo (at most 32 W)
  int4 hcm[32 * W];                       // coarse nodes of the halo vertices
  float4 rc[kDsmCoarseBanks * BANK];      // coarse-level inputs (first level pushed)
  float4 zc[kDsmCoarseBanks * BANK];      // coarse-level outputs
  __nv_bfloat16 rb[W][8][BANK];           // BF16 apply: residual as B operand
  float4 zs[W][BANK];                     // BF16 apply / split bank rows
  double red[W][3];
  double part[kDsmMaxCtas][kDsmPartSlots];  // partials of every CTA (pushed)
  float4 zown[32 * W];                    // fine-level z of the own slots
  float4 hzs[32 * W];                     // fine-level z of the halo (pushed by the owners)
  int push[kDsmPushPerThread * 32 * W];   // this CTA's pushes (own slot, CTA, halo index)
  // Coarse-level bookkeeping staged once per solve: per coarse bank its real
  // slots; per node of a level above the first, first member | member count
  // << 16 (members: rc indices of the level below).
  int gval[kDsmCoarseBanks];
  int mnode[kDsmCoarseBanks * BANK];
  int mem[kDsmCoarseBanks * BANK];
  unsigned tmem_base;  // tensor-memory address of the CTA's row store
};

__device__ __forceinline__ void stage_bank_full(const MasLevelDev& lv, int bank, float* slot,
                                                int lane) {
  const float* src = lv.M + (size_t)bank * kPacked;
  for (int e = lane; e < kDsmBankFloats; e += 32)
    slot[e] = src[upper_index(BANK, e & (BANK - 1), e >> 5)];
  __syncwarp();
}

// z (lane row) = M r over columns [k0, k1) of a full column-major bank, with
// the residuals read as shared-memory broadcasts: the products of
// bank_apply_smem summed in the same order.
__device__ __forceinline__ float3 bank_apply_full(const float* M, const float4* rs, int lane,
                                                  int k0, int k1) {
  float zx = 0.f, zy = 0.f, zz = 0.f;
#pragma unroll 8
  for (int k = k0; k < k1; ++k) {
    float m = M[k * BANK + lane];
    float4 rk = rs[k];
    zx += m * rk.x;
    zy += m * rk.y;
    zz += m * rk.z;
  }
  return make_float3(zx, zy, zz);
}

// Off-diagonal row sum plus the diagonal term, every column in shared memory.
__device__ __forceinline__ float3 dsm_row(const int2* e, int rw, const float4* pl, float d,
                                          float3 pv) {
  float yx = d * pv.x, yy = d * pv.y, yz = d * pv.z;
#pragma unroll 4
  for (int j = 0; j < rw; ++j) {
    int2 q = e[j * BANK];
    float val = __int_as_float(q.y);
    float4 pj = pl[-1 - q.x];
    yx = fmaf(val, pj.x, yx);
    yy = fmaf(val, pj.y, yy);
    yz = fmaf(val, pj.z, yz);
  }
  return make_float3(yx, yy, yz);
}

// dsm_row with the row entries read from tensor memory, eight per load (the
// entries of dsm_row in the same order, so the same sums).
// 48 columns (24 entries) of this thread's lane in flight at once, one wait.
__device__ __forceinline__ void tmem_ld48_wait(unsigned taddr, unsigned (&v)[48]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%48];\n"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, "
      "%41, %42, %43, %44, %45, %46, %47}, [%49];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]),
        "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]),
        "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47])
      : "r"(taddr), "r"(taddr + 32u)
      : "memory");
}

__device__ __forceinline__ float3 dsm_row_tmem(unsigned taddr, int rw, int tm_rw,
                                               const float4* pl, float d, float3 pv) {
  float yx = d * pv.x, yy = d * pv.y, yz = d * pv.z;
  if (rw <= 24 && tm_rw >= 24) {
    // The whole row behind one wait (rw is the same in the warp; the warp's
    // columns hold at least 24 entries, so the 48 read are its own).
    unsigned e[48];
    tmem_ld48_wait(taddr, e);
#pragma unroll
    for (int k = 0; k < 24; ++k) {
      if (k < rw) {
        const float val = __uint_as_float(e[2 * k + 1]);
        const float4 pj = pl[-1 - (int)e[2 * k]];
        yx = fmaf(val, pj.x, yx);
        yy = fmaf(val, pj.y, yy);
        yz = fmaf(val, pj.z, yz);
      }
    }
    return make_float3(yx, yy, yz);
  }
  for (int j0 = 0; j0 < rw; j0 += 8) {
    unsigned e[16];
    tmem_ld16_wait(taddr + 2 * j0, e);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (j0 + k < rw) {
        const float val = __uint_as_float(e[2 * k + 1]);
        const float4 pj = pl[-1 - (int)e[2 * k]];
        yx = fmaf(val, pj.x, yx);
        yy = fmaf(val, pj.y, yy);
        yz = fmaf(val, pj.z, yz);
      }
    }
  }
  return make_float3(yx, yy, yz);
}

template <int F>
__global__ void __launch_bounds__(32 * F, 1) cg_dsm_cluster_kernel(CgArgs a) {
  if (a.skip && *a.skip) return;  // the ADMM solve already ended (every CTA alike)
  constexpr int W = F, T = 32 * F;
  extern __shared__ __align__(16) unsigned char dsm_smem[];
  DsmShared<W>& s = *reinterpret_cast<DsmShared<W>*>(dsm_smem);
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = blockIdx.x, nctas = gridDim.x;
  const int fb = q * F + warp;
  const bool bank_ok = fb < a.nbank0;
  const int levels = a.levels;
  const bool tc = a.bf16 != 0;
  CgTrace tr(a.trace, 2);
  int iter = -1;

  // Bank offsets of the coarse levels in Mc / rc / zc.
  int cbo[MAX_COARSE + 1];
  cbo[0] = 0;
#pragma unroll
  for (int l = 0; l < MAX_COARSE; ++l) cbo[l + 1] = cbo[l] + (l < levels ? a.coarse[l].nbank : 0);
  const int ncb = cbo[levels];
  int cnode[MAX_COARSE];  // real nodes per coarse level
#pragma unroll
  for (int l = 0; l < MAX_COARSE; ++l) cnode[l] = l < levels ? a.coarse[l].nnode : 0;
  auto stage = [&](const MasLevelDev& lv, int bank, float* slot) {
    if (tc)
      stage_bank_frag(lv, bank, slot, lane);
    else
      stage_bank_full(lv, bank, slot, lane);
  };
  // Store this CTA's N block sums t[] into slots slot0.. of every CTA's
  // s.part row q.
  auto push_partials = [&](int slot0, const double* t, int N) {
    if (warp == 0 && lane < nctas) {
      double* dst = cl.map_shared_rank(&s.part[q][slot0], lane);
      for (int k = 0; k < N; ++k) dst[k] = t[k];
    }
  };
  // Sum of one partial slot over the CTAs: a warp sum in a fixed lane order,
  // the same in every warp of every CTA.
  auto total = [&](int slot) {
    return warp_sum_d(lane < nctas ? s.part[lane][slot] : 0.0);
  };
  // Block sum of N doubles per thread into t[] of every thread: warp sums
  // into s.red, one block barrier, then every warp sums the warps' values
  // with the same butterfly (identical totals in all warps, in a fixed
  // order).  The next write of s.red comes after a later block or cluster
  // barrier.
  auto block_sum = [&](const double* v, int N, double* t) {
    for (int k = 0; k < N; ++k) {
      double x = warp_sum_d(v[k]);
      if (lane == 0) s.red[warp][k] = x;
    }
    __syncthreads();
    for (int k = 0; k < N; ++k) t[k] = warp_sum_d(lane < W ? s.red[lane][k] : 0.0);
  };

  // ---- one-time staging ----------------------------------------------------
  for (int i = lane; i < 5 * BANK; i += 32) s.rb[warp][3 + i / BANK][i % BANK] = __float2bfloat16_rn(0.f);
  int vbase = 0, vsize = 0, rptr = 0, rw = 0;
  if (bank_ok) {
    vbase = a.part_off[fb];
    vsize = a.part_off[fb + 1] - vbase;
    rptr = a.rb_ptr[fb];
    rw = a.rb_w[fb];
    stage(a.fine, fb, s.Mf[warp]);
  }
#pragma unroll
  for (int l = 0; l < MAX_COARSE; ++l) {
    if (l >= levels) break;
    for (int g = cbo[l] + warp; g < cbo[l + 1]; g += W) {
      stage(a.coarse[l], g - cbo[l], s.Mc[g]);
      if (lane == 0) s.gval[g] = min(max(cnode[l] - (g - cbo[l]) * BANK, 0), BANK);
    }
    if (l >= 1) {
      // Members of level l's nodes, after those of the levels below.
      int base = 0;
#pragma unroll
      for (int k = 1; k < MAX_COARSE; ++k)
        if (k < l) base += a.coarse[k].member_off[cnode[k]];
      const MasLevelDev& lv = a.coarse[l];
      for (int nd = tid; nd < cnode[l]; nd += T) {
        const int m0 = lv.member_off[nd], m1 = lv.member_off[nd + 1];
        s.mnode[cbo[l] * BANK + nd] = (base + m0) | ((m1 - m0) << 16);
        for (int m = m0; m < m1; ++m) s.mem[base + m] = cbo[l - 1] * BANK + lv.member[m];
      }
    }
  }
  for (int i = tid; i < kDsmCoarseBanks * BANK; i += T) {
    s.rc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    s.zc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  const bool own = lane < vsize;
  const int v = vbase + lane;
  const int2* erow = a.rent + rptr + lane;
  float d = 0.f;
  float3 x = make_float3(0.f, 0.f, 0.f), b = x;
  int cm[MAX_COARSE] = {0, 0, 0, 0};
  if (own) {
    d = a.Ldiag[v] + a.dyn[v];
    float4 x4 = a.x[v], b4 = a.b[v];
    x = make_float3(x4.x, x4.y, x4.z);
    b = make_float3(b4.x, b4.y, b4.z);
    int4 c = a.cmap[v];
    cm[0] = c.x;
    cm[1] = c.y;
    cm[2] = c.z;
    cm[3] = c.w;
  }
  int hcol = -1;
  {
    const int h0 = a.halo_off[q], nh = a.halo_off[q + 1] - h0;
    if (tid < nh) {
      hcol = a.halo_col[h0 + tid];
      s.hcm[tid] = a.cmap[hcol];
    }
  }
  const int npush = a.push_off[q + 1] - a.push_off[q];
  for (int i = tid; i < npush; i += T) s.push[i] = a.push[a.push_off[q] + i];
  // Row store in tensor memory: warp w keeps its bank's rows in lanes
  // 32 (w % 4).. and columns 2 tm_rw (w / 4) .. 2 tm_rw (w / 4 + 1) - 1,
  // entries past the bank's width padded with (own slot, 0) and never read.
  const bool tm = a.tm_cols > 0 && (W / 4) * 2 * a.tm_rw <= a.tm_cols && rw <= a.tm_rw;
  unsigned taddr = 0;
  if (a.tm_cols > 0) {
    if (warp == 0) tmem_alloc(&s.tmem_base, (unsigned)a.tm_cols);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    taddr = s.tmem_base + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)((warp >> 2) * 2 * a.tm_rw);
    if (tm) {
      for (int j0 = 0; j0 < rw; j0 += 8) {
        unsigned e[16];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int2 qe = j0 + k < rw ? erow[(j0 + k) * BANK] : make_int2(-1 - tid, 0);
          e[2 * k] = (unsigned)qe.x;
          e[2 * k + 1] = (unsigned)qe.y;
        }
        tmem_st16_wait(taddr + 2 * j0, e);
      }
    }
  }
  auto row = [&](float3 pv) {
    return tm ? dsm_row_tmem(taddr, rw, a.tm_rw, s.pl, d, pv) : dsm_row(erow, rw, s.pl, d, pv);
  };
  // Every warp's tensor-memory accesses are complete before warp 0 frees it.
  auto tm_release = [&]() {
    if (a.tm_cols <= 0) return;
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
      tmem_fence_after();
      tmem_dealloc(s.tmem_base, (unsigned)a.tm_cols);
    }
  };
  auto gather_halo = [&](const float4* ex) {
    if (hcol >= 0) s.pl[T + tid] = ldcg4(ex + hcol);
    __syncthreads();
  };
  // z of a vertex: fine-level z plus the coarse z of its node at every level,
  // in level order (the same operations for an own and a halo vertex).
  auto full_z = [&](float3 z, int c0, int c1, int c2, int c3) {
    const int c[MAX_COARSE] = {c0, c1, c2, c3};
#pragma unroll
    for (int l = 0; l < MAX_COARSE; ++l) {
      if (l >= levels) break;
      float4 qz = s.zc[cbo[l] * BANK + c[l]];
      z.x += qz.x;
      z.y += qz.y;
      z.z += qz.z;
    }
    return z;
  };

  // Publish x for r = b - A x; the cluster barrier also guarantees that every
  // CTA has finished staging before any CTA stores into its shared memory.
  s.pl[tid] = make_float4(x.x, x.y, x.z, 0.f);
  if (own) a.p[v] = make_float4(x.x, x.y, x.z, 0.f);
  cl.sync();
  gather_halo(a.p);
  float3 r;
  {
    float3 y = row(x);
    r = own ? make_float3(b.x - y.x, b.y - y.y, b.z - y.z) : make_float3(0.f, 0.f, 0.f);
  }
  double rr_plain0 = -1.0;
  if (a.x_alt) {
    float3 xa = make_float3(0.f, 0.f, 0.f);
    if (own) {
      float4 qa = a.x_alt[v];
      xa = make_float3(qa.x, qa.y, qa.z);
    }
    __syncthreads();
    s.pl[tid] = make_float4(xa.x, xa.y, xa.z, 0.f);
    if (own) a.Ap[v] = make_float4(xa.x, xa.y, xa.z, 0.f);
    cl.sync();
    gather_halo(a.Ap);
    float3 ra;
    {
      float3 y = row(xa);
      ra = own ? make_float3(b.x - y.x, b.y - y.y, b.z - y.z) : make_float3(0.f, 0.f, 0.f);
    }
    const double v3[3] = {(double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z,
                          (double)r.x * ra.x + (double)r.y * ra.y + (double)r.z * ra.z,
                          (double)ra.x * ra.x + (double)ra.y * ra.y + (double)ra.z * ra.z};
    double t3[3];
    block_sum(v3, 3, t3);
    push_partials(3, t3, 3);
    cl.sync();
    const double rr_plain = total(3), r_pa = total(4), rr_alt = total(5);
    rr_plain0 = rr_plain;
    const float w = (float)blend_weight(rr_plain, r_pa, rr_alt);
    if (w > 0.0f) {
      x = make_float3(x.x + w * (xa.x - x.x), x.y + w * (xa.y - x.y), x.z + w * (xa.z - x.z));
      r = make_float3(r.x + w * (ra.x - r.x), r.y + w * (ra.y - r.y), r.z + w * (ra.z - r.z));
      if (q == 0 && tid == 0 && a.stats) atomicAdd(a.stats + a.alt_stat, 1);
    }
  }

  // Phase C body: fine MAS of r, pushes of the first-level input and of the
  // r.z / r.r partials, fine z published for the halos.
  float3 z0 = make_float3(0.f, 0.f, 0.f), p = z0, Ap = z0;
  float4 hz = make_float4(0.f, 0.f, 0.f, 0.f);
  auto mas_fine = [&]() {
    const double rr = own ? (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z : 0.0;
    __syncwarp();
    if (!bank_ok) {
      z0 = make_float3(0.f, 0.f, 0.f);
    } else if (tc) {
      z0 = bank_apply_mma(s.Mf[warp], r, lane, s.rb[warp], s.zs[warp]);
    } else {
      // The warp's residuals go through its own slots of pl, which nothing
      // reads between the SpMV and the next p update.
      s.pl[tid] = make_float4(r.x, r.y, r.z, 0.f);
      __syncwarp();
      z0 = bank_apply_full(s.Mf[warp], s.pl + warp * BANK, lane, 0, BANK);
    }
    if (!own) z0 = make_float3(0.f, 0.f, 0.f);
    const double rz = own ? (double)r.x * z0.x + (double)r.y * z0.y + (double)r.z * z0.z : 0.0;
    tr.stamp(iter, 6);
    if (levels > 0) {
      const float sx = warp_sum(r.x), sy = warp_sum(r.y), sz = warp_sum(r.z);
      if (bank_ok && lane < nctas) {
        float4* dst = cl.map_shared_rank(&s.rc[fb], lane);
        *dst = make_float4(sx, sy, sz, 0.f);
      }
    }
    s.zown[tid] = make_float4(z0.x, z0.y, z0.z, 0.f);
    const double v2[2] = {rz, rr};
    double t2[2];
    block_sum(v2, 2, t2);  // its barrier also publishes zown to the CTA
    push_partials(0, t2, 2);
    for (int i = tid; i < npush; i += T) {
      const int e = s.push[i];
      float4* dst = cl.map_shared_rank(&s.hzs[e >> 15], (e >> 10) & 31);
      *dst = s.zown[e & 1023];
    }
    tr.stamp(iter, 7);
  };
  // Phase A head: totals and every coarse level.
  auto totals = [&](double& rz, double& rr) {
    rz = total(0);
    rr = total(1);
    if (levels == 0) return;
    tr.stamp(iter, 9);
    // Restriction chain: one warp per node of the next level sums its
    // members (at most 32, one per lane) with a warp sum.
#pragma unroll
    for (int l = 1; l < MAX_COARSE; ++l) {
      if (l >= levels) break;
      for (int nd = warp; nd < cnode[l]; nd += W) {
        const int e = s.mnode[cbo[l] * BANK + nd];
        const int m0 = e & 0xffff, cnt = e >> 16;
        float4 qv = lane < cnt ? s.rc[s.mem[m0 + lane]] : make_float4(0.f, 0.f, 0.f, 0.f);
        float qx = warp_sum(qv.x), qy = warp_sum(qv.y), qz = warp_sum(qv.z);
        if (lane == 0) s.rc[cbo[l] * BANK + nd] = make_float4(qx, qy, qz, 0.f);
      }
      __syncthreads();
    }
    tr.stamp(iter, 10);
    // Every coarse bank: BF16 one warp per bank on the tensor cores; FP32 the
    // columns of a bank split over `split` warps, partial rows added by the
    // bank's first warp in warp order.
    double rzc = 0.0;
    const int split = tc ? 1 : (ncb * 4 <= W ? 4 : (ncb * 2 <= W ? 2 : 1));
    const int per_round = W / split;
    for (int g0 = 0; g0 < ncb; g0 += per_round) {
      const int g = g0 + warp / split, part = warp - (warp / split) * split;
      const bool gok = g < ncb;
      const bool gvalid = gok && lane < s.gval[g];
      const int slot = g * BANK + lane;
      if (tc) {
        if (gok) {
          float4 qv = s.rc[slot];
          float3 rl = gvalid ? make_float3(qv.x, qv.y, qv.z) : make_float3(0.f, 0.f, 0.f);
          float3 zq = bank_apply_mma(s.Mc[g], rl, lane, s.rb[warp], s.zs[warp]);
          if (!gvalid) zq = make_float3(0.f, 0.f, 0.f);
          s.zc[slot] = make_float4(zq.x, zq.y, zq.z, 0.f);
          rzc += (double)rl.x * zq.x + (double)rl.y * zq.y + (double)rl.z * zq.z;
        }
      } else {
        if (gok) {
          const int cols = BANK / split, k0 = part * cols;
          float3 zp = bank_apply_full(s.Mc[g], s.rc + g * BANK, lane, k0, k0 + cols);
          s.zs[warp][lane] = make_float4(zp.x, zp.y, zp.z, 0.f);
        }
        __syncthreads();
        if (gok && part == 0) {
          float4 acc = s.zs[warp][lane];
          for (int k = 1; k < split; ++k) {
            float4 t = s.zs[warp + k][lane];
            acc.x += t.x;
            acc.y += t.y;
            acc.z += t.z;
          }
          float4 qv = s.rc[slot];
          float3 rl = gvalid ? make_float3(qv.x, qv.y, qv.z) : make_float3(0.f, 0.f, 0.f);
          float3 zq = gvalid ? make_float3(acc.x, acc.y, acc.z) : make_float3(0.f, 0.f, 0.f);
          s.zc[slot] = make_float4(zq.x, zq.y, zq.z, 0.f);
          rzc += (double)rl.x * zq.x + (double)rl.y * zq.y + (double)rl.z * zq.z;
        }
        // s.zs is reused by the next round; after the last one the block sum's
        // barrier publishes s.zc.
        if (g0 + per_round < ncb) __syncthreads();
      }
    }
    tr.stamp(iter, 11);
    const double v1[1] = {rzc};
    double t1[1];
    block_sum(v1, 1, t1);
    rz += t1[0];
    tr.stamp(iter, 12);
  };

  __syncthreads();  // every warp has read pl in the residual rows
  mas_fine();
  cl.sync();
  if (hcol >= 0) hz = s.hzs[tid];
  double rz, rr;
  totals(rz, rr);
  iter = 0;
  if (!isfinite(rz)) {
    if (q == 0 && tid == 0) {
      a.result[0] = 0;
      a.result[1] = kCgInvalidInitialResidual;
      *a.result_rr = (float)rr;
    }
    tm_release();
    return;  // every CTA takes the same decision; no store is in flight
  }
  const double rr0 = rr_plain0 >= 0.0 ? rr_plain0 : rr;
  const double abs2 = (double)a.abs_tol * a.abs_tol;
  const float rel_tol = a.rel_tol_dev ? *a.rel_tol_dev : a.rel_tol;
  const double rel2 = (double)rel_tol * rel_tol;
  double beta = 0.0;
  int status = kCgMaxIter;
  while (true) {
    {
      const float bt = (float)beta;
      float3 zt = full_z(z0, cm[0], cm[1], cm[2], cm[3]);
      p = bt == 0.0f ? zt : make_float3(zt.x + bt * p.x, zt.y + bt * p.y, zt.z + bt * p.z);
      if (!own) p = make_float3(0.f, 0.f, 0.f);
      s.pl[tid] = make_float4(p.x, p.y, p.z, 0.f);
      if (hcol >= 0) {
        const int4 c4 = s.hcm[tid];
        float3 zh = full_z(make_float3(hz.x, hz.y, hz.z), c4.x, c4.y, c4.z, c4.w);
        float4 po = s.pl[T + tid];
        float3 ph = bt == 0.0f ? zh
                               : make_float3(zh.x + bt * po.x, zh.y + bt * po.y, zh.z + bt * po.z);
        s.pl[T + tid] = make_float4(ph.x, ph.y, ph.z, 0.f);
      }
    }
    tr.stamp(iter, 0);
    __syncthreads();
    tr.stamp(iter, 1);
    {
      Ap = row(p);
      if (!own) Ap = make_float3(0.f, 0.f, 0.f);
      tr.stamp(iter, 2);
      const double v1[1] = {own ? (double)p.x * Ap.x + (double)p.y * Ap.y + (double)p.z * Ap.z
                                : 0.0};
      double t1[1];
      block_sum(v1, 1, t1);
      push_partials(2, t1, 1);
    }
    tr.stamp(iter, 3);
    cl.sync();
    tr.stamp(iter, 4);
    {
      const double pAp = total(2);
      tr.stamp(iter, 5);
      const float alpha = (float)(fabs(pAp) < 1e-20 ? 0.0 : rz / pAp);
      x = make_float3(alpha * p.x + x.x, alpha * p.y + x.y, alpha * p.z + x.z);
      r = make_float3(-alpha * Ap.x + r.x, -alpha * Ap.y + r.y, -alpha * Ap.z + r.z);
      if (!own) r = make_float3(0.f, 0.f, 0.f);
      mas_fine();
    }
    cl.sync();
    tr.stamp(iter, 8);
    if (hcol >= 0) hz = s.hzs[tid];
    const double rz_old = rz;
    totals(rz, rr);
    tr.stamp(iter, 13);
    ++iter;
    bool stop = false;
    if (iter >= a.max_iter) {
      status = kCgMaxIter;
      stop = true;
    } else if (rr <= abs2) {
      status = kCgAbsTol;
      stop = true;
    } else if (rr <= rel2 * rr0) {
      status = kCgRelTol;
      stop = true;
    }
    beta = fabs(rz_old) < 1e-20 ? 0.0 : rz / rz_old;
    if (stop) break;
  }
  tm_release();
  if (own) a.x[v] = make_float4(x.x, x.y, x.z, 0.f);
  tr.finish(iter);
  if (q == 0 && tid == 0) {
    a.result[0] = iter;
    a.result[1] = status;
    *a.result_rr = (float)rr;
    if (a.stats) {
      atomicAdd(a.stats, iter);
      atomicAdd(a.stats + 1, 1);
      if (a.first_solve) atomicAdd(a.stats + 2, iter);
    }
  }
}

template <int F>
size_t dsm_smem_bytes() {
  return sizeof(DsmShared<F>);
}

template <int F>
int dsm_max_cluster() {
  static const int n = [] {
    const size_t smem = sizeof(DsmShared<F>);
    if (cudaFuncSetAttribute(cg_dsm_cluster_kernel<F>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(cg_dsm_cluster_kernel<F>,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kDsmMaxCtas);
    cfg.blockDim = dim3(32 * F);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kDsmMaxCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int m = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&m, cg_dsm_cluster_kernel<F>, &cfg) != cudaSuccess) {
      cudaGetLastError();
      m = 0;
    }
    return m < kDsmMaxCtas ? m : kDsmMaxCtas;
  }();
  return n;
}

template <int F>
void launch_dsm(const CgArgs& a, int nctas, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nctas);
  cfg.blockDim = dim3(32 * F);
  cfg.dynamicSmemBytes = sizeof(DsmShared<F>);
  cfg.stream = st;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = nctas;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  CUDA_CHECK(cudaLaunchKernelEx(&cfg, cg_dsm_cluster_kernel<F>, a));
  SILK_LAUNCHED();
}

}  // namespace

void launch_galerkin_fill(const GalerkinDev& g, const double* src_vals,
                          const float* dyn, cudaStream_t st) {
  if (g.n_entries == 0) return;
  galerkin_fill_kernel<<<div_up(g.n_entries, 256), 256, 0, st>>>(g, src_vals, dyn);
  SILK_LAUNCHED();
}

void launch_bank_invert(const MasLevelDev& lv, bool fine, const int* part_off,
                        const double* src_vals, const float* dyn, int* fail,
                        cudaStream_t st) {
  if (lv.nbank == 0) return;
  bank_invert_kernel<<<lv.nbank, 256, 0, st>>>(lv, fine ? 1 : 0, part_off,
                                               src_vals, dyn, fail);
  SILK_LAUNCHED();
}

int cg_grid_size(int nslices, int nbank0) {
  int want_blocks = div_up(nslices > nbank0 ? nslices : nbank0, kCgWarps);
  int cl = max_cluster_size();
  // One cluster while each warp has at most ~3 slices / banks to process.
  if (cl > 0 && want_blocks <= 3 * cl) return -cl;
  static const int max_coop = [] {
    int dev = 0, sms = 0, per_sm = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    size_t smem = kCgWarps * kPacked * sizeof(float);
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_kernel,
                                                             kCgThreads, smem));
    return sms * (per_sm > 0 ? per_sm : 1);
  }();
  int want = div_up(nslices > nbank0 ? nslices : nbank0, kCgWarps);
  if (want < 1) want = 1;
  return want < max_coop ? want : max_coop;
}

void launch_cg(const CgArgs& a, int grid, cudaStream_t st) {
  size_t smem = kCgWarps * kPacked * sizeof(float);
  if (grid < 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(-grid);
    cfg.blockDim = dim3(kCgThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = -grid;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    CUDA_CHECK(cudaLaunchKernelEx(&cfg, cg_kernel_cluster, a));
    SILK_LAUNCHED();
    return;
  }
  CUDA_CHECK(cudaMemsetAsync(a.barrier, 0, 2 * sizeof(unsigned), st));
  void* args[] = {(void*)&a};
  CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)cg_kernel, dim3(grid),
                                         dim3(kCgThreads), args, smem, st));
  SILK_LAUNCHED();
}

int cg_resident_grid(int res_blocks) {
  struct Limits {
    int max_coop = 0, max_cluster = 0;
  };
  static const Limits lim = [] {
    Limits l;
    const size_t smem = sizeof(ResShared);
    int dev = 0, sms = 0, per_sm = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CUDA_CHECK(cudaFuncSetAttribute(cg_resident_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CUDA_CHECK(cudaFuncSetAttribute(cg_resident_cluster_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_resident_kernel, kResThreads,
                                                      smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
    l.max_coop = sms * per_sm;
    if (cudaFuncSetAttribute(cg_resident_cluster_kernel,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      cudaGetLastError();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kResThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 16;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&n, cg_resident_cluster_kernel, &cfg) !=
        cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    l.max_cluster = n >= 16 ? 16 : (n >= 8 ? 8 : 0);
    return l;
  }();
  if (res_blocks <= 0 || lim.max_coop == 0) return 0;
  if (res_blocks > 1 && res_blocks <= lim.max_cluster) return -res_blocks;
  return res_blocks <= lim.max_coop ? res_blocks : 0;
}

void launch_cg_resident(const CgArgs& a, int grid, cudaStream_t st) {
  const size_t smem = sizeof(ResShared);
  if (grid < 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(-grid);
    cfg.blockDim = dim3(kResThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = -grid;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    CUDA_CHECK(cudaLaunchKernelEx(&cfg, cg_resident_cluster_kernel, a));
    SILK_LAUNCHED();
    return;
  }
  CUDA_CHECK(cudaMemsetAsync(a.barrier, 0, 2 * sizeof(unsigned), st));
  void* args[] = {(void*)&a};
  CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)cg_resident_kernel, dim3(grid),
                                         dim3(kResThreads), args, smem, st));
  SILK_LAUNCHED();
}

int cg_dsm_ctas(int nbank0, int f) {
  if (nbank0 <= 0 || (f != 8 && f != 16)) return 0;
  const int nctas = div_up(nbank0, f);
  const int cap = f == 8 ? dsm_max_cluster<8>() : dsm_max_cluster<16>();
  return nctas >= 2 && nctas <= cap ? nctas : 0;
}

void launch_cg_dsm(const CgArgs& a, int nctas, cudaStream_t st) {
  if (a.dsm_f == 8)
    launch_dsm<8>(a, nctas, st);
  else
    launch_dsm<16>(a, nctas, st);
}

}  // namespace silkb
