// Tensor-memory-accelerator (TMA) tile loads of one level of a 3-D field
// [nz][ny][P] into shared memory, completing on an mbarrier.
//
// Host: level_map() encodes a tensor map (float32, dims P x ny x nz, strides
// P*4 and ny*P*4 bytes, box BX x BY x 1, out-of-bounds elements read as 0)
// through the driver's cuTensorMapEncodeTiled (fetched once with
// cudaGetDriverEntryPoint, so the library does not link libcuda).
// Device: mbarrier init / expect-tx / bounded parity wait, and the 3-D tiled
// bulk copy.  Rules the callers keep: the box's innermost extent is a
// multiple of 4 floats (16 bytes) and every x coordinate is a multiple of 4;
// the shared destination is 128-byte aligned; a tensor map covers this GPU's
// own memory only, and no copy uses cluster multicast.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace zm {

// Encode the map of a [nz][ny][P] float32 field with a BX x BY x 1 box; false
// if the driver refused (the caller reports the error).
bool level_map(CUtensorMap* map, const float* base, int P, int ny, int nz, int bx, int by);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false if it did not
// complete within max_polls tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned max_polls) {
  const uint32_t a = smem_u32(bar);
  for (unsigned n = 0; n < max_polls; ++n) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One BX x BY tile of level z at (x, y) (x a multiple of 4; x, y may lie
// outside the field, where the tile reads zeros).
__device__ __forceinline__ void tma_level(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace zm
