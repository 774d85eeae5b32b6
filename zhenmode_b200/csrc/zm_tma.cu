// Host side of the TMA level maps (see zm_tma.cuh).
#include <cudaTypedefs.h>

#include <mutex>

#include "zm_tma.cuh"

namespace zm {

namespace {
PFN_cuTensorMapEncodeTiled g_encode = nullptr;
std::once_flag g_once;
}  // namespace

bool level_map(CUtensorMap* map, const float* base, int P, int ny, int nz, int bx, int by) {
  std::call_once(g_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  });
  if (!g_encode || (P % 4) != 0 || (bx % 4) != 0 || (reinterpret_cast<uintptr_t>(base) % 16) != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)P * 4, (cuuint64_t)P * ny * 4};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace zm
