// Learned CG warm start: feature extraction, the forward on the
// 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory,
// FP32 accumulators in tensor memory; for training it also keeps the
// pre-activations and the output gradient), the backward pass (FP32,
// straight through the BF16 rounding) with deterministic per-block gradient
// partials, and the Adam update.  No counterpart in the reference.
#include <cuda_bf16.h>

#include "learned.cuh"

namespace silkb {

namespace {

constexpr int kBwdThreads = 256;
constexpr int kBwdTile = 32;  // samples per backward tile
constexpr int kBwdBlocks = 296;

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) +
         x * expf(-0.5f * x * x) * 0.39894228040143268f;
}
__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

// ---------------------------------------------------------------------------
// Forward on the 5th-generation tensor cores: a CTA of 256 threads carries
// tiles of 128 samples through the four layers as
// tcgen05.mma.cta_group::1.kind::f16 products (M = 128, BF16 operands from
// shared memory, FP32 accumulators in 64 tensor-memory columns), one thread
// issuing each layer's K / 16 products and committing them to an mbarrier;
// warps w and w + 4 then read the 32 accumulator lanes of quarter w % 4
// (tcgen05.ld 32x32b), each half of the columns, add the bias, apply GELU and
// write the next layer's A operand as BF16.
// Operands are K-major without swizzle: 8 x 8 BF16 core matrices of 128 B,
// adjacent along K (leading byte offset 128) and K / 8 apart along M or N
// (stride byte offset).  The rounding points of the model (BF16
// layer inputs and weights, FP32 sums, bias added to the sum, as the CPU
// oracle's forward); the order of the FP32 additions inside a product is the
// tensor core's.
constexpr int kTcRows = 128;
constexpr int kTcThreads = 256;             // two warps per 32-lane quarter of the accumulators
constexpr int kTcCols = 64;                 // tensor-memory columns (N <= 64)
constexpr int kTcOutN = 16;                 // output layer padded to N = 16
constexpr long long kTcWaitSpins = 1 << 20; // mbarrier polls before giving up

// The B operands of the four layers, in the order and layout they take in
// shared memory (the weight image, prepared once per parameter vector).
struct TcWeights {
  __nv_bfloat16 w1[kMlpH * kMlpK];      // B of layer 1: N 64, K 16
  __nv_bfloat16 w2[kMlpH * kMlpH];      // N 64, K 64
  __nv_bfloat16 w3[kMlpH * kMlpH];
  __nv_bfloat16 w4[kTcOutN * kMlpH];    // N 16 (8..15 zero), K 64
};
static_assert(sizeof(TcWeights) % 128 == 0 && sizeof(TcWeights) == 2 * kMlpWeightImage,
              "one bulk copy of 16-byte units");

struct TcSmem {
  alignas(128) TcWeights w;
  alignas(128) __nv_bfloat16 a[kTcRows * kMlpH];     // A: M 128, K 16 or 64
  float bias[3 * kMlpH + kMlpKOut];
  float mean[kMlpK], inv_std[kMlpK];
  alignas(8) uint64_t bar;   // the layers' products
  alignas(8) uint64_t wbar;  // the weight image's bulk copy
  unsigned tmem;
};

// Element index of (row r, column k) in a K-major core-matrix layout of
// width K.
__device__ __forceinline__ int cm_index(int r, int k, int K) {
  return (((r >> 3) * (K >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}
__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
// Shared-memory matrix descriptor (no swizzle, descriptor version 1).
__device__ __forceinline__ uint64_t umma_desc(const void* p, unsigned lbo, unsigned sbo) {
  return (uint64_t)((su32(p) & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: F32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(unsigned d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(bar))
               : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* bar, unsigned parity) {
  for (long long i = 0; i < kTcWaitSpins; ++i)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 16 accumulator columns of this thread's lane; the wait is in the same
// statement, so no use of the outputs is scheduled before it.
__device__ __forceinline__ void tc_ld16(unsigned taddr, float (&v)[16]) {
  unsigned u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]),
        "=r"(u[7]), "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]),
        "=r"(u[14]), "=r"(u[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(u[j]);
}

// kTrain: rows index[r] (or r) of feat / t_hat, the hidden pre-activations
// stored (z[l][r][64], stride n), the output gradient d4 = 2 (o - t) / (3n)
// (n x 8, columns >= 3 zero) and a per-block loss partial instead of out.
// Weight image: B(n, k) = W[k][n] of each layer in BF16, K-major core
// matrices (the output layer's columns 8..15 zero).
__global__ void mlp_image_kernel(const float* __restrict__ P, TcWeights* __restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kMlpH * kMlpK) {
    const int nn = i / kMlpK, k = i % kMlpK;
    img->w1[cm_index(nn, k, kMlpK)] = __float2bfloat16_rn(P[kOffW1 + k * kMlpH + nn]);
  }
  if (i < kMlpH * kMlpH) {
    const int nn = i / kMlpH, k = i % kMlpH;
    img->w2[cm_index(nn, k, kMlpH)] = __float2bfloat16_rn(P[kOffW2 + k * kMlpH + nn]);
    img->w3[cm_index(nn, k, kMlpH)] = __float2bfloat16_rn(P[kOffW3 + k * kMlpH + nn]);
  }
  if (i < kTcOutN * kMlpH) {
    const int nn = i / kMlpH, k = i % kMlpH;
    img->w4[cm_index(nn, k, kMlpH)] =
        __float2bfloat16_rn(nn < kMlpKOut ? P[kOffW4 + k * kMlpKOut + nn] : 0.0f);
  }
}

// kTrain: rows index[r] (or r) of feat / t_hat, the hidden pre-activations
// stored (z[l][r][64], stride n), the output gradient d4 = 2 (o - t) / (3n)
// (n x 8, columns >= 3 zero) and a per-block loss partial instead of out.
template <bool kTrain>
__global__ void __launch_bounds__(kTcThreads) mlp_forward_tc_kernel(
    MlpDev m, const float* __restrict__ feat, int n, float* __restrict__ out,
    int* __restrict__ fail, const float* __restrict__ t_hat, const int* __restrict__ index,
    float* __restrict__ z, float* __restrict__ d4, double* __restrict__ loss_part) {
  extern __shared__ __align__(128) unsigned char tc_raw[];
  TcSmem& s = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int quarter = warp & 3, half = warp >> 2;  // accumulator lanes and column half
  // The weight image arrives by one bulk copy; biases and statistics by
  // plain loads meanwhile.
  const float* P = m.params;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&s.bar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&s.wbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(&s.wbar)),
                 "r"((unsigned)sizeof(TcWeights))
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(su32(&s.w)), "l"(m.image), "r"((unsigned)sizeof(TcWeights)), "r"(su32(&s.wbar))
        : "memory");
  }
  for (int i = tid; i < kMlpH; i += kTcThreads) {
    s.bias[i] = P[kOffB1 + i];
    s.bias[kMlpH + i] = P[kOffB2 + i];
    s.bias[2 * kMlpH + i] = P[kOffB3 + i];
  }
  if (tid < kMlpKOut) s.bias[3 * kMlpH + tid] = P[kOffB4 + tid];
  if (tid < kMlpK) {
    s.mean[tid] = P[kOffMean + tid];
    s.inv_std[tid] = 1.0f / P[kOffStd + tid];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&s.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  bool ok = __syncthreads_and(bar_wait(&s.wbar, 0u)) != 0;
  const unsigned tmem = s.tmem;
  const unsigned taddr = tmem + ((unsigned)(quarter * 32) << 16);  // this warp's 32 lanes
  unsigned phase = 0, commits = 0;
  // One layer's products: D (128 x N) = A (128 x K) B^T, then wait for them.
  auto layer_mma = [&](const __nv_bfloat16* w, int K, int N) {
    if (tid == 0) {
      tc_fence_after();
      const unsigned sbo = (unsigned)(K / 8) * 128u;
      for (int kc = 0; kc < K / 16; ++kc)
        umma_bf16(tmem, umma_desc(s.a + kc * 128, 128u, sbo), umma_desc(w + kc * 128, 128u, sbo),
                  umma_idesc(kTcRows, N), kc > 0 ? 1u : 0u);
      umma_commit(&s.bar);
    }
    ++commits;
    const bool done = bar_wait(&s.bar, phase);
    phase ^= 1u;
    tc_fence_after();
    return __syncthreads_and(done) != 0;
  };
  const int ntiles = (n + kTcRows - 1) / kTcRows;
  const float scale = 2.0f / (3.0f * (float)n);
  double loss = 0.0;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int r = quarter * 32 + (tid & 31), row = tile * kTcRows + r;
    const int src = row < n ? (kTrain && index ? index[row] : row) : -1;
    // Layer-1 input: normalised features in BF16 (rows past n are zero), this
    // thread's half of its row's 16.
    {
      const int c0 = 8 * half;
      float x[8];
#pragma unroll
      for (int c = 0; c < 8; ++c)
        x[c] = src >= 0 ? (feat[(size_t)src * kMlpK + c0 + c] - s.mean[c0 + c]) * s.inv_std[c0 + c]
                        : 0.0f;
      uint4 q;
      q.x = pack_bf16(x[0], x[1]);
      q.y = pack_bf16(x[2], x[3]);
      q.z = pack_bf16(x[4], x[5]);
      q.w = pack_bf16(x[6], x[7]);
      *reinterpret_cast<uint4*>(s.a + cm_index(r, c0, kMlpK)) = q;
    }
    proxy_fence();
    __syncthreads();
    const __nv_bfloat16* ws[3] = {s.w.w1, s.w.w2, s.w.w3};
    for (int l = 0; l < 3 && ok; ++l) {
      ok = layer_mma(ws[l], l == 0 ? kMlpK : kMlpH, kMlpH);
      if (!ok) break;
      // Bias, GELU, BF16: the next layer's A (K = 64) from this thread's row.
#pragma unroll
      for (int cc = 0; cc < kMlpH / 2; cc += 16) {
        const int c0 = (kMlpH / 2) * half + cc;
        float v[16];
        tc_ld16(taddr + c0, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += s.bias[l * kMlpH + c0 + j];
        if (kTrain && row < n) {
          float4* zr = reinterpret_cast<float4*>(z + (size_t)l * n * kMlpH + (size_t)row * kMlpH + c0);
#pragma unroll
          for (int j = 0; j < 16; j += 4) zr[j / 4] = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
        uint4 q[2];
        uint32_t* qw = reinterpret_cast<uint32_t*>(q);
#pragma unroll
        for (int j = 0; j < 16; j += 2) qw[j / 2] = pack_bf16(gelu(v[j]), gelu(v[j + 1]));
        *reinterpret_cast<uint4*>(s.a + cm_index(r, c0, kMlpH)) = q[0];
        *reinterpret_cast<uint4*>(s.a + cm_index(r, c0 + 8, kMlpH)) = q[1];
      }
      tc_fence_before();
      proxy_fence();
      __syncthreads();
    }
    if (!ok) break;
    ok = layer_mma(s.w.w4, kMlpH, kTcOutN);
    if (!ok) break;
    float v[16];
    if (half == 0) tc_ld16(taddr, v);  // warp-uniform: warps 0-3 hold the 16 output columns
    if (half == 0 && row < n) {
      if constexpr (kTrain) {
#pragma unroll
        for (int c = 0; c < kMlpKOut; ++c) {
          float dv = 0.0f;
          if (c < kMlpOut) {
            const float e = (v[c] + s.bias[3 * kMlpH + c]) - t_hat[(size_t)src * 4 + c];
            loss += (double)e * e;
            dv = scale * e;
          }
          d4[(size_t)row * kMlpKOut + c] = dv;
        }
      } else {
#pragma unroll
        for (int c = 0; c < kMlpOut; ++c)
          out[(size_t)row * kMlpOut + c] = v[c] + s.bias[3 * kMlpH + c];
      }
    }
    tc_fence_before();
    __syncthreads();  // every lane's accumulators read before the next tile's products
  }
  if constexpr (kTrain) {
    // Loss partial of this block, in a fixed order (warp sums, then warps).
    __shared__ double red[kTcThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, off);
    if ((tid & 31) == 0) red[warp] = loss;
    __syncthreads();
    if (tid == 0) {
      double a = 0.0;
      for (int w = 0; w < kTcThreads / 32; ++w) a += red[w];
      loss_part[blockIdx.x] = a;
    }
  }
  if (!ok) {
    // A copy or product did not complete in time: report it and wait
    // (bounded) for what is still in flight before the tensor memory is freed.
    if (tid == 0 && fail) atomicOr(fail, kFailMlpWait);
    bar_wait(&s.wbar, 0u);
    if (commits > 0u) bar_wait(&s.bar, phase ^ 1u);  // the last commit's phase
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcCols)
                 : "memory");
  }
}

struct BwdSmem {
  float W[3][kMlpH][kMlpH + 1];  // BF16-rounded W2, W3 and (first 8 columns) W4
  float A[kBwdTile][kMlpH + 1];  // layer input of the current layer (rounded)
  float D[kBwdTile][kMlpH + 1];  // output gradient of the current layer
  float E[kBwdTile][kMlpH + 1];  // gradient propagated to the layer input
};

// Backward over tiles of 32 samples: per-block partial gradients of every
// trainable parameter (layout of the parameter vector), summed later in a
// fixed order.
__global__ void __launch_bounds__(kBwdThreads) mlp_backward_kernel(
    MlpDev m, const float* __restrict__ feat, const int* __restrict__ index, int n,
    const float* __restrict__ z, const float* __restrict__ d4, float* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char bwd_raw[];
  BwdSmem& s = *reinterpret_cast<BwdSmem*>(bwd_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kMlpH * kMlpH; i += kBwdThreads) {
    int r = i / kMlpH, c = i % kMlpH;
    s.W[0][r][c] = bf16r(m.params[kOffW2 + i]);
    s.W[1][r][c] = bf16r(m.params[kOffW3 + i]);
    s.W[2][r][c] = c < kMlpKOut ? bf16r(m.params[kOffW4 + r * kMlpKOut + c]) : 0.0f;
  }
  // Accumulators: dW4 (512), dW3 (4096), dW2 (4096), dW1 (1024), biases.
  float gW4[2] = {0.f, 0.f}, gW3[16], gW2[16], gW1[4] = {0.f, 0.f, 0.f, 0.f};
  float gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gb4 = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) gW3[k] = gW2[k] = 0.f;
  __syncthreads();
  const int ntiles = (n + kBwdTile - 1) / kBwdTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int s0 = tile * kBwdTile;
    // Output layer: D = d4, A = bf16(gelu(z3)).
    for (int i = tid; i < kBwdTile * kMlpH; i += kBwdThreads) {
      int r = i / kMlpH, c = i % kMlpH, sidx = s0 + r;
      bool ok = sidx < n;
      s.A[r][c] = ok ? bf16r(gelu(z[(size_t)2 * n * kMlpH + (size_t)sidx * kMlpH + c])) : 0.f;
      s.D[r][c] = (ok && c < kMlpKOut) ? d4[(size_t)sidx * kMlpKOut + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      int e = tid + kBwdThreads * k, i = e / kMlpKOut, j = e % kMlpKOut;
      float acc = 0.f;
      for (int r = 0; r < kBwdTile; ++r) acc += s.A[r][i] * s.D[r][j];
      gW4[k] += acc;
    }
    if (tid < kMlpKOut)
      for (int r = 0; r < kBwdTile; ++r) gb4 += s.D[r][tid];
    // Hidden layers 3, 2, 1 (l = 2, 1, 0): E = D W^T of the layer above,
    // D_l = E * gelu'(z_l), A_l = layer input.
    for (int l = 2; l >= 0; --l) {
      const int wi = l;  // W[l] holds the weights of layer l + 1 (W2 for l = 0)
      const int kout = (l == 2) ? kMlpKOut : kMlpH;
      __syncthreads();
      for (int i = tid; i < kBwdTile * kMlpH; i += kBwdThreads) {
        int r = i / kMlpH, c = i % kMlpH;
        float acc = 0.f;
        for (int j = 0; j < kout; ++j) acc += s.D[r][j] * s.W[wi][c][j];
        int sidx = s0 + r;
        float zz = sidx < n ? z[(size_t)l * n * kMlpH + (size_t)sidx * kMlpH + c] : 0.f;
        s.E[r][c] = sidx < n ? acc * gelu_grad(zz) : 0.f;
      }
      __syncthreads();
      // Layer input of hidden layer l: bf16(gelu(z_{l-1})) or the normalised
      // features for l = 0.
      for (int i = tid; i < kBwdTile * kMlpH; i += kBwdThreads) {
        int r = i / kMlpH, c = i % kMlpH, sidx = s0 + r;
        float v = 0.f;
        if (sidx < n) {
          if (l > 0) {
            v = bf16r(gelu(z[(size_t)(l - 1) * n * kMlpH + (size_t)sidx * kMlpH + c]));
          } else if (c < kMlpK) {
            int src = index ? index[sidx] : sidx;
            v = bf16r((feat[(size_t)src * kMlpK + c] - m.params[kOffMean + c]) /
                      m.params[kOffStd + c]);
          }
        }
        s.A[r][c] = v;
      }
      __syncthreads();
      if (l > 0) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          int e = tid + kBwdThreads * k, i = e / kMlpH, j = e % kMlpH;
          float acc = 0.f;
          for (int r = 0; r < kBwdTile; ++r) acc += s.A[r][i] * s.E[r][j];
          if (l == 2) gW3[k] += acc; else gW2[k] += acc;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          int e = tid + kBwdThreads * k, i = e / kMlpH, j = e % kMlpH;
          float acc = 0.f;
          for (int r = 0; r < kBwdTile; ++r) acc += s.A[r][i] * s.E[r][j];
          gW1[k] += acc;
        }
      }
      if (tid < kMlpH) {
        float acc = 0.f;
        for (int r = 0; r < kBwdTile; ++r) acc += s.E[r][tid];
        if (l == 2) gb3 += acc; else if (l == 1) gb2 += acc; else gb1 += acc;
      }
      __syncthreads();
      // The propagated gradient becomes the output gradient of the layer below.
      for (int i = tid; i < kBwdTile * kMlpH; i += kBwdThreads) {
        int r = i / kMlpH, c = i % kMlpH;
        s.D[r][c] = s.E[r][c];
      }
    }
    __syncthreads();
  }
  float* out = part + (size_t)blockIdx.x * kMlpTrainParams;
#pragma unroll
  for (int k = 0; k < 2; ++k) out[kOffW4 + tid + kBwdThreads * k] = gW4[k];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    out[kOffW3 + tid + kBwdThreads * k] = gW3[k];
    out[kOffW2 + tid + kBwdThreads * k] = gW2[k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) out[kOffW1 + tid + kBwdThreads * k] = gW1[k];
  if (tid < kMlpH) {
    out[kOffB1 + tid] = gb1;
    out[kOffB2 + tid] = gb2;
    out[kOffB3 + tid] = gb3;
  }
  if (tid < kMlpKOut) out[kOffB4 + tid] = gb4;
}

__global__ void mlp_reduce_kernel(const float* __restrict__ part, int nblocks,
                                  const double* __restrict__ loss_part, int nloss,
                                  double inv_count, float* __restrict__ grad,
                                  double* __restrict__ loss_out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    float acc = 0.f;
    if (p < kMlpTrainParams)
      for (int b = 0; b < nblocks; ++b) acc += part[(size_t)b * kMlpTrainParams + p];
    grad[p] = acc;
  }
  if (p == 0) {
    double a = 0.0;
    for (int b = 0; b < nloss; ++b) a += loss_part[b];
    *loss_out = a * inv_count;
  }
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                                float* __restrict__ m, float* __restrict__ v, float lr,
                                float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpTrainParams) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float gi = g[i];
  float mi = b1 * m[i] + (1.0f - b1) * gi;
  float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

__global__ void warm_features_kernel(int n, const float4* __restrict__ x0,
                                     const float4* __restrict__ x1,
                                     const float4* __restrict__ x2,
                                     const float4* __restrict__ y,
                                     const uint8_t* __restrict__ pin,
                                     const int* __restrict__ ring_off,
                                     const int* __restrict__ ring, float inv_sigma,
                                     float* __restrict__ feat) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  float4 a = x0[v], b = x1[v], c = x2[v], p = y[v];
  float mx = 0.f, my = 0.f, mz = 0.f;
  int beg = ring_off[v], end = ring_off[v + 1];
  for (int q = beg; q < end; ++q) {
    int u = ring[q];
    float4 ua = x0[u], ub = x1[u];
    mx += ua.x - ub.x;
    my += ua.y - ub.y;
    mz += ua.z - ub.z;
  }
  float inv_cnt = end > beg ? 1.0f / (float)(end - beg) : 0.0f;
  float4* f = reinterpret_cast<float4*>(feat + (size_t)v * kMlpK);
  f[0] = make_float4((p.x - a.x) * inv_sigma, (p.y - a.y) * inv_sigma, (p.z - a.z) * inv_sigma,
                     (a.x - b.x) * inv_sigma);
  f[1] = make_float4((a.y - b.y) * inv_sigma, (a.z - b.z) * inv_sigma, (b.x - c.x) * inv_sigma,
                     (b.y - c.y) * inv_sigma);
  f[2] = make_float4((b.z - c.z) * inv_sigma, mx * inv_cnt * inv_sigma, my * inv_cnt * inv_sigma,
                     mz * inv_cnt * inv_sigma);
  f[3] = make_float4(pin[v] ? 1.0f : 0.0f, 0.f, 0.f, 0.f);
}

__global__ void warm_combine_kernel(int n, const float* __restrict__ o,
                                    const float* __restrict__ params,
                                    const float4* __restrict__ y, float sigma,
                                    float4* __restrict__ xp) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  float4 b = y[v];
  xp[v] = make_float4(b.x + sigma * params[kOffOutScale] * o[3 * v],
                      b.y + sigma * params[kOffOutScale + 1] * o[3 * v + 1],
                      b.z + sigma * params[kOffOutScale + 2] * o[3 * v + 2], 0.f);
}

__global__ void warm_target_kernel(int n, const float4* __restrict__ x,
                                   const float4* __restrict__ y, float inv_sigma,
                                   float* __restrict__ t) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  float4 a = x[v], b = y[v];
  reinterpret_cast<float4*>(t)[v] =
      make_float4((a.x - b.x) * inv_sigma, (a.y - b.y) * inv_sigma, (a.z - b.z) * inv_sigma, 0.f);
}

// Learned iterate start (CG solves of ADMM iterations >= 3): scale of the
// last ADMM step, sigma = sqrt(mean |x_k - x_(k-1)|^2) over the vertices
// (one block, FP64 sum in a fixed order), floored so the features stay finite.
__global__ void __launch_bounds__(1024) iterate_scale_kernel(int n, const float4* __restrict__ x,
                                                             const float4* __restrict__ h1,
                                                             float* __restrict__ sigma) {
  __shared__ double part[32];
  double acc = 0.0;
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    float4 a = x[v], b = h1[v];
    float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    acc += (double)dx * dx + (double)dy * dy + (double)dz * dz;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *sigma = fmaxf((float)sqrt(t / (double)(n > 0 ? n : 1)), 1e-20f);
  }
}

// Features of the iterate model: the last two ADMM steps x_k - x_(k-1) and
// x_(k-1) - x_(k-2), their 1-ring means (all over sigma) and the pin flag.
__global__ void iterate_features_kernel(int n, const float4* __restrict__ x,
                                        const float4* __restrict__ h1,
                                        const float4* __restrict__ h2,
                                        const uint8_t* __restrict__ pin,
                                        const int* __restrict__ ring_off,
                                        const int* __restrict__ ring,
                                        const float* __restrict__ sigma,
                                        float* __restrict__ feat) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const float is = 1.0f / *sigma;
  float4 a = x[v], b = h1[v], c = h2[v];
  float m1x = 0.f, m1y = 0.f, m1z = 0.f, m2x = 0.f, m2y = 0.f, m2z = 0.f;
  int beg = ring_off[v], end = ring_off[v + 1];
  for (int q = beg; q < end; ++q) {
    int u = ring[q];
    float4 ua = x[u], ub = h1[u], uc = h2[u];
    m1x += ua.x - ub.x;
    m1y += ua.y - ub.y;
    m1z += ua.z - ub.z;
    m2x += ub.x - uc.x;
    m2y += ub.y - uc.y;
    m2z += ub.z - uc.z;
  }
  const float ic = (end > beg ? 1.0f / (float)(end - beg) : 0.0f) * is;
  float4* f = reinterpret_cast<float4*>(feat + (size_t)v * kMlpK);
  f[0] = make_float4((a.x - b.x) * is, (a.y - b.y) * is, (a.z - b.z) * is, (b.x - c.x) * is);
  f[1] = make_float4((b.y - c.y) * is, (b.z - c.z) * is, m1x * ic, m1y * ic);
  f[2] = make_float4(m1z * ic, m2x * ic, m2y * ic, m2z * ic);
  f[3] = make_float4(pin[v] ? 1.0f : 0.0f, 0.f, 0.f, 0.f);
}

// x_pred = x + sigma * out_scale * MLP output.
__global__ void iterate_combine_kernel(int n, const float* __restrict__ o,
                                       const float* __restrict__ params,
                                       const float4* __restrict__ x,
                                       const float* __restrict__ sigma,
                                       float4* __restrict__ xp) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const float sg = *sigma;
  float4 b = x[v];
  xp[v] = make_float4(b.x + sg * params[kOffOutScale] * o[3 * v],
                      b.y + sg * params[kOffOutScale + 1] * o[3 * v + 1],
                      b.z + sg * params[kOffOutScale + 2] * o[3 * v + 2], 0.f);
}

// Training samples of the iterate model: m vertices (a stride through the
// mesh, shifted by `salt` from one iteration to the next) with their
// features and target (x_new - x_old) / sigma, appended while the buffer has
// room (the counter keeps counting).
__global__ void iterate_sample_kernel(int m, int n, unsigned salt, const float* __restrict__ feat,
                                      const float4* __restrict__ x_new,
                                      const float4* __restrict__ x_old,
                                      const float* __restrict__ sigma,
                                      float* __restrict__ out_feat, float* __restrict__ out_tgt,
                                      int* __restrict__ counter, int cap,
                                      const int* __restrict__ skip) {
  if (skip && *skip) return;  // the ADMM solve already ended: no iterate to sample
  __shared__ int base;
  if (threadIdx.x == 0) base = atomicAdd(counter, m);
  __syncthreads();
  const float is = 1.0f / *sigma;
  const unsigned stride = (unsigned)(n / m > 1 ? n / m : 1);
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const int slot = base + j;
    if (slot >= cap) return;
    const int v = (int)((salt + (unsigned)j * stride) % (unsigned)n);
    const float4* fs = reinterpret_cast<const float4*>(feat + (size_t)v * kMlpK);
    float4* fd = reinterpret_cast<float4*>(out_feat + (size_t)slot * kMlpK);
    for (int k = 0; k < kMlpK / 4; ++k) fd[k] = fs[k];
    float4 a = x_new[v], b = x_old[v];
    reinterpret_cast<float4*>(out_tgt)[slot] =
        make_float4((a.x - b.x) * is, (a.y - b.y) * is, (a.z - b.z) * is, 0.f);
  }
}


}  // namespace


// Persistent grid of the tensor-core forward: one CTA per 128-sample tile, at
// most 4 per SM (256 threads, ~37 KB of shared memory and 64 tensor-memory
// columns each).
int tc_grid(int n) {
  static const int max_grid = [] {
    int dev = 0, sms = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return 4 * sms;
  }();
  const int tiles = (n + kTcRows - 1) / kTcRows;
  return tiles < 1 ? 1 : (tiles < max_grid ? tiles : max_grid);
}

void mlp_image(const float* params, uint16_t* image, cudaStream_t st) {
  mlp_image_kernel<<<div_up(kMlpH * kMlpH, 256), 256, 0, st>>>(
      params, reinterpret_cast<TcWeights*>(image));
  SILK_LAUNCHED();
}

void mlp_forward(const MlpDev& m, const float* feat, int n, float* out, cudaStream_t st) {
  if (n <= 0) return;
  mlp_forward_tc_kernel<false><<<tc_grid(n), kTcThreads, sizeof(TcSmem), st>>>(
      m, feat, n, out, m.fail, nullptr, nullptr, nullptr, nullptr, nullptr);
  SILK_LAUNCHED();
}

size_t mlp_work_floats(int n) {
  // z (3 x n x 64) + d4 (n x 8) + backward partials + loss partials (doubles).
  return (size_t)3 * n * kMlpH + (size_t)n * kMlpKOut +
         (size_t)kBwdBlocks * kMlpTrainParams + 2 * (size_t)tc_grid(n) + 4;
}

void mlp_loss_grad(const MlpDev& m, const float* feat, const float* t_hat, int n,
                   const int* index, float* work, float* grad, double* loss_out,
                   cudaStream_t st) {
  float* z = work;
  float* d4 = z + (size_t)3 * n * kMlpH;
  float* part = d4 + (size_t)n * kMlpKOut;
  size_t off = (size_t)3 * n * kMlpH + (size_t)n * kMlpKOut + (size_t)kBwdBlocks * kMlpTrainParams;
  off = (off + 1) & ~(size_t)1;  // 8-byte alignment for the doubles
  double* loss_part = reinterpret_cast<double*>(work + off);
  const int fg = tc_grid(n);
  mlp_forward_tc_kernel<true><<<fg, kTcThreads, sizeof(TcSmem), st>>>(
      m, feat, n, nullptr, m.fail, t_hat, index, z, d4, loss_part);
  SILK_LAUNCHED();
  static const bool attr = [] {
    CUDA_CHECK(cudaFuncSetAttribute(mlp_backward_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(BwdSmem)));
    return true;
  }();
  (void)attr;
  mlp_backward_kernel<<<kBwdBlocks, kBwdThreads, sizeof(BwdSmem), st>>>(m, feat, index, n, z, d4,
                                                                        part);
  SILK_LAUNCHED();
  mlp_reduce_kernel<<<div_up(kMlpParams, 128), 128, 0, st>>>(
      part, kBwdBlocks, loss_part, fg, 1.0 / (3.0 * n), grad, loss_out);
  SILK_LAUNCHED();
}

void mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr,
              cudaStream_t st) {
  float c1 = 1.0f / (1.0f - powf(0.9f, (float)step));
  float c2 = 1.0f / (1.0f - powf(0.999f, (float)step));
  mlp_adam_kernel<<<div_up(kMlpTrainParams, 256), 256, 0, st>>>(params, grad, m, v, lr, c1, c2);
  SILK_LAUNCHED();
}

void warm_features(int n, const float4* x0, const float4* x1, const float4* x2,
                   const float4* y, const uint8_t* pin, const int* ring_off,
                   const int* ring, float inv_sigma, float* feat, cudaStream_t st) {
  if (n <= 0) return;
  warm_features_kernel<<<div_up(n, 256), 256, 0, st>>>(n, x0, x1, x2, y, pin, ring_off, ring,
                                                       inv_sigma, feat);
  SILK_LAUNCHED();
}

void warm_predict(const MlpDev& m, int n, const float* feat, const float4* y, float sigma,
                  float* out_tmp, float4* x_pred, cudaStream_t st) {
  if (n <= 0) return;
  mlp_forward(m, feat, n, out_tmp, st);
  warm_combine_kernel<<<div_up(n, 256), 256, 0, st>>>(n, out_tmp, m.params, y, sigma, x_pred);
  SILK_LAUNCHED();
}

void warm_target(int n, const float4* x, const float4* y, float inv_sigma, float* t,
                 cudaStream_t st) {
  if (n <= 0) return;
  warm_target_kernel<<<div_up(n, 256), 256, 0, st>>>(n, x, y, inv_sigma, t);
  SILK_LAUNCHED();
}

void iterate_predict(const MlpDev& m, int n, const float4* x, const float4* h1, const float4* h2,
                     const uint8_t* pin, const int* ring_off, const int* ring, float* sigma,
                     float* feat, float* out_tmp, float4* x_pred, cudaStream_t st) {
  if (n <= 0) return;
  iterate_scale_kernel<<<1, 1024, 0, st>>>(n, x, h1, sigma);
  SILK_LAUNCHED();
  iterate_features_kernel<<<div_up(n, 256), 256, 0, st>>>(n, x, h1, h2, pin, ring_off, ring, sigma,
                                                          feat);
  SILK_LAUNCHED();
  if (!m.params) return;  // features only (sample capture without a model)
  mlp_forward(m, feat, n, out_tmp, st);
  iterate_combine_kernel<<<div_up(n, 256), 256, 0, st>>>(n, out_tmp, m.params, x, sigma, x_pred);
  SILK_LAUNCHED();
}

void iterate_samples(int m, int n, unsigned salt, const float* feat, const float4* x_new,
                     const float4* x_old, const float* sigma, float* out_feat, float* out_tgt,
                     int* counter, int cap, const int* skip, cudaStream_t st) {
  if (n <= 0 || m <= 0) return;
  iterate_sample_kernel<<<1, 256, 0, st>>>(m, n, salt, feat, x_new, x_old, sigma, out_feat,
                                           out_tgt, counter, cap, skip);
  SILK_LAUNCHED();
}

}  // namespace silkb

