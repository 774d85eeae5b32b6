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

__device__ __forceinline__ unsigned atom_inc_acq_rel(unsigned* p, unsigned wrap) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.inc.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(wrap) : "memory");
  return old;
}

__device__ __forceinline__ void red_add_release(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The barrier generation this block waits past, kept by its thread 0.
__device__ __forceinline__ unsigned& barrier_gen() {
  __shared__ unsigned gen;
  return gen;
}

// Every kernel that uses grid_barrier calls this first (all blocks): thread 0
// reads the generation word once.  No barrier can complete before every block
// has arrived at it, so the value read is the one the first barrier advances.
__device__ __forceinline__ void grid_barrier_begin(const unsigned* bar) {
  if (threadIdx.x == 0) barrier_gen() = ld_acquire(bar + 1);
}

// Grid-wide barrier over co-resident blocks: bar[0] counts arrivals and wraps
// to 0 at the last one (atom.inc), which then advances the generation bar[1]
// with release semantics; the others poll the generation with acquire loads
// (the error word every 256 polls).  Returns false (and sets *err) if the wait
// exceeded its poll limit or another block reported an error.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned* err, unsigned nblocks, unsigned max_polls) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    unsigned& my_gen = barrier_gen();
    // release: this block's writes (ordered before by __syncthreads) are
    // visible to whoever acquires the counter or, through the last arrival,
    // the generation
    if (atom_inc_acq_rel(bar, nblocks - 1) == nblocks - 1) {
      red_add_release(bar + 1, 1u);
    } else {
      unsigned polls = 0;
      while (ld_acquire(bar + 1) == my_gen) {
        if (++polls > max_polls || ((polls & 255u) == 0u && ld_acquire(err) != 0u)) {
          atomicOr(err, ZM_BT_ERR_BARRIER);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    ++my_gen;
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace zm
