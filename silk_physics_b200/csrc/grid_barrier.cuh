// Grid-wide barrier for cooperative launches, with a bounded wait: when the
// spin limit runs out the barrier records an error and every block leaves at
// its next barrier, so a kernel can never wait forever.
#pragma once

#include <cuda/atomic>

namespace silkb {

constexpr long long kBarrierSpinLimit = 1ll << 25;  // ~2 s with back-off

struct GridBarrier {
  unsigned* count;
  unsigned* err;
  unsigned* gen;
  unsigned nblocks;

  __device__ bool sync() {
    __shared__ int s_ok;
    if (nblocks == 1u) {
      __syncthreads();
      return true;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> g(*gen), c(*count),
          e(*err);
      int ok = 1;
      unsigned my = g.load(cuda::memory_order_relaxed);
      if (e.load(cuda::memory_order_relaxed) != 0u) {
        ok = 0;
      } else {
        unsigned arrived = c.fetch_add(1u, cuda::memory_order_acq_rel);
        if (arrived == nblocks - 1u) {
          c.store(0u, cuda::memory_order_relaxed);
          g.fetch_add(1u, cuda::memory_order_release);
        } else {
          long long spins = 0;
          while (g.load(cuda::memory_order_acquire) == my) {
            if (e.load(cuda::memory_order_relaxed) != 0u) {
              ok = 0;
              break;
            }
            if (++spins > kBarrierSpinLimit) {
              e.store(1u, cuda::memory_order_relaxed);
              ok = 0;
              break;
            }
            __nanosleep(32);
          }
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  }
};

}  // namespace silkb
