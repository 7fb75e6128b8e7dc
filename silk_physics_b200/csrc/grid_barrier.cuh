// Grid-wide barrier for cooperative launches, with a bounded wait: when the
// spin limit runs out the barrier records an error and every block leaves at
// its next barrier, so a kernel can never wait forever.
#pragma once

#include <cuda/atomic>

namespace silkb {

constexpr long long kBarrierSpinLimit = 1ll << 22;  // polls: ~2-4 s (an L2 round trip each)

// The k-th barrier of a launch waits until the arrival counter (zero at
// launch, never reset) reaches k x nblocks: one atomic per block on the
// critical path and no generation word for the last block to bump.
struct GridBarrier {
  unsigned* count;
  unsigned* err;
  unsigned* unused;
  unsigned nblocks;
  unsigned epoch = 0;  // barriers passed by this block
  long long limit = kBarrierSpinLimit;  // polls before the wait gives up
  // Failure-detection tests only: this block never arrives, so the others'
  // waits run out (it waits, bounded by the same limit, for their error).
  unsigned withhold = 0xffffffffu;

  __device__ bool sync() {
    __shared__ int s_ok;
    if (nblocks == 1u) {
      __syncthreads();
      return true;
    }
    ++epoch;
    __syncthreads();
    if (threadIdx.x == 0) {
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> c(*count), e(*err);
      int ok = 1;
      if (e.load(cuda::memory_order_relaxed) != 0u) {
        ok = 0;
      } else if (blockIdx.x == withhold) {
        long long spins = 0;
        while (e.load(cuda::memory_order_relaxed) == 0u && ++spins <= limit) __nanosleep(32);
        e.store(1u, cuda::memory_order_relaxed);
        ok = 0;
      } else {
        const unsigned target = epoch * nblocks;
        unsigned arrived = c.fetch_add(1u, cuda::memory_order_acq_rel) + 1u;
        long long spins = 0;
        while (arrived < target) {
          if (e.load(cuda::memory_order_relaxed) != 0u) {
            ok = 0;
            break;
          }
          if (++spins > limit) {
            e.store(1u, cuda::memory_order_relaxed);
            ok = 0;
            break;
          }
          __nanosleep(32);
          arrived = c.load(cuda::memory_order_acquire);
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  }
};

}  // namespace silkb
