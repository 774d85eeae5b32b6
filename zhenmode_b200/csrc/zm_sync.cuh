// Grid-wide barrier of the cooperative kernels (barotropic subcycle, column
// projection).  Every wait is bounded: a block that polls longer than its
// limit, or sees another block's error, records ZM_BT_ERR_BARRIER and returns
// false, and the kernel then returns from every block.
#pragma once

#include "zm_kernels.cuh"

namespace zm {

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier over co-resident blocks: arrival counter + generation.
// Returns false (and sets *err) if the wait exceeded its poll limit.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned* err, unsigned nblocks, unsigned max_polls) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    unsigned* count = bar;
    unsigned* gen = bar + 1;
    const unsigned my_gen = ld_acquire(gen);
    __threadfence();
    const unsigned arrived = atomicAdd(count, 1u);
    if (arrived == nblocks - 1) {
      *count = 0u;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      unsigned polls = 0;
      while (ld_acquire(gen) == my_gen) {
        if (++polls > max_polls || ld_acquire(err) != 0u) {
          atomicOr(err, ZM_BT_ERR_BARRIER);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace zm
