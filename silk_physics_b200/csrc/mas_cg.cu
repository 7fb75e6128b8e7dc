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
//    fixed order by every block).
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
// Galerkin operator, virtual slots are identity).
__global__ void __launch_bounds__(256) bank_invert_kernel(
    MasLevelDev lv, int fine, const int* part_off, const double* src_vals,
    const float* dyn) {
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

template <class Barrier>
__device__ __forceinline__ void cg_body(const CgArgs& a, Barrier& bar, float* sm_all) {
  double* part = a.partials + 4 * blockIdx.x;
  // r = b - A x.
  spmv_phase(a, a.x, a.r, 1);
  if (!bar.sync()) return;
  {
    double v[2] = {0.0, 0.0};
    fine_phase(a, 0.f, false, sm_all, v[0], v[1]);
    block_sum<2>(v, part);
  }
  if (!bar.sync()) return;
  if (blockIdx.x == 0) {
    double v[1] = {coarse_phase(a, sm_all)};
    block_sum<1>(v, a.coarse_partial);
  }
  if (!bar.sync()) return;
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
  const double rr0 = rr;
  const double abs2 = (double)a.abs_tol * a.abs_tol;
  const double rel2 = (double)a.rel_tol * a.rel_tol;
  double beta = 0.0;
  int iter = 0;
  int status = kCgMaxIter;
  while (true) {
    prolong_phase(a, (float)beta);
    if (!bar.sync()) return;
    {
      double v[1] = {spmv_phase(a, a.p, a.Ap, 0)};
      block_sum<1>(v, part + 2);
    }
    if (!bar.sync()) return;
    double pAp = grid_total(a.partials, 2, gridDim.x);
    double alpha = fabs(pAp) < 1e-20 ? 0.0 : rz / pAp;
    {
      double v[2] = {0.0, 0.0};
      fine_phase(a, (float)alpha, true, sm_all, v[0], v[1]);
      block_sum<2>(v, part);
    }
    if (!bar.sync()) return;
    if (blockIdx.x == 0) {
      double v[1] = {coarse_phase(a, sm_all)};
      block_sum<1>(v, a.coarse_partial);
    }
    if (!bar.sync()) return;
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
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.result[0] = iter;
    a.result[1] = status;
    *a.result_rr = (float)rr;
    if (a.stats) {
      atomicAdd(a.stats, iter);
      atomicAdd(a.stats + 1, 1);
    }
  }
}

__global__ void __launch_bounds__(kCgThreads) cg_kernel(CgArgs a) {
  extern __shared__ float sm_all[];
  GridBarrier bar{a.barrier, a.barrier + 1, a.barrier + 2, gridDim.x};
  cg_body(a, bar, sm_all);
}

__global__ void __launch_bounds__(kCgThreads) cg_kernel_cluster(CgArgs a) {
  extern __shared__ float sm_all[];
  ClusterBarrier bar;
  cg_body(a, bar, sm_all);
}

int max_cluster_size() {
  static int size = -1;
  if (size < 0) {
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
    size = n >= 16 ? 16 : (n >= 8 ? 8 : 0);
  }
  return size;
}

}  // namespace

void launch_galerkin_fill(const GalerkinDev& g, const double* src_vals,
                          const float* dyn, cudaStream_t st) {
  if (g.n_entries == 0) return;
  galerkin_fill_kernel<<<div_up(g.n_entries, 256), 256, 0, st>>>(g, src_vals, dyn);
  SILK_LAUNCHED();
}

void launch_bank_invert(const MasLevelDev& lv, bool fine, const int* part_off,
                        const double* src_vals, const float* dyn,
                        cudaStream_t st) {
  if (lv.nbank == 0) return;
  bank_invert_kernel<<<lv.nbank, 256, 0, st>>>(lv, fine ? 1 : 0, part_off,
                                               src_vals, dyn);
  SILK_LAUNCHED();
}

int cg_grid_size(int nslices, int nbank0) {
  int want_blocks = div_up(nslices > nbank0 ? nslices : nbank0, kCgWarps);
  int cl = max_cluster_size();
  // One cluster while each warp has at most ~3 slices / banks to process.
  if (cl > 0 && want_blocks <= 3 * cl) return -cl;
  static int max_coop = 0;
  if (max_coop == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    size_t smem = kCgWarps * kPacked * sizeof(float);
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_kernel,
                                                             kCgThreads, smem));
    max_coop = sms * (per_sm > 0 ? per_sm : 1);
  }
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

}  // namespace silkb
